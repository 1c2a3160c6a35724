// Reduced-precision form: BF16 tensor-core screen (tcgen05, FP32 accumulate
// in TMEM) into a widened candidate list of k' per query, FP32 re-rank from
// the original vectors with the reference's arithmetic (distance.h:62-72),
// FP64 recompute of the candidates within 1e-6 relative of the k-th FP32
// distance so the boundary order follows exact arithmetic.
//
// Layouts (both operands K-major, no swizzle, core matrices of 8 rows x 16 B):
//   query tile A: 128 queries x 112 bf16, element (q, k) at
//                 ((k/8)*16 + q/8)*64 + (q%8)*8 + k%8
//   row block  B: 128 rows x 112 bf16, same formula with the row index
// Dims 0..99 carry the vector; on the row side dims 100/101 carry
// -|x|^2/2 split into a bf16 high part and a bf16 remainder, on the query
// side dims 100/101 are 1.0.  The MMA therefore produces
// acc = q.x - |x|^2/2, and ds = |q|^2 - 2*acc approximates |q - x|^2 with no
// per-row term left for the epilogue: a row is a candidate for query q iff
// acc >= (|q|^2 - T_q)/2, one compare per TMEM value.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "tc_util.cuh"

namespace fknn {

namespace {

constexpr int BQ = 128;                       // queries per tile = MMA M = TMEM lanes
constexpr int BR = 128;                       // rows per sub-tile = MMA N
constexpr int BS = 2;                         // shared-memory stages for row blocks
constexpr int B_EPI_WARPS = 4;
constexpr int B_THREADS = (2 + B_EPI_WARPS) * 32;  // producer, MMA issuer, 4 epilogue warps
constexpr uint32_t TMEM_COLS = 2 * BR;        // double-buffered accumulator
constexpr int STAGE_ROW = 36;                 // floats per lane row of the push staging area

// Operand formats of the tensor-core screen.  Both operands are K-major,
// no swizzle, in core matrices of 8 rows x 16 bytes; every MMA consumes 32
// bytes of K per row (two core-matrix columns), so the descriptors of both
// formats are alike and only the MMA kind, its K and the bytes per row differ.
struct FmtBF16 {
  static constexpr bool kFP8 = false;
  static constexpr int K = 112;                 // 100 dims, 2 norm terms, zero padding
  static constexpr int ROW_BYTES = K * 2;
  static constexpr int MMAS = K / 16;           // kind::f16: K = 16 per MMA
  // F32 accumulate, BF16 A and B, K-major, N = BR, M = BQ
  static constexpr uint32_t IDESC =
      (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BR >> 3) << 17) | ((uint32_t)(BQ >> 4) << 24);
};
struct FmtFP8 {
  static constexpr bool kFP8 = true;
  static constexpr int K = 128;                 // 100 dims, 3 norm terms, zero padding
  static constexpr int ROW_BYTES = K;
  static constexpr int MMAS = K / 32;           // kind::f8f6f4: K = 32 per MMA
  // F32 accumulate, E4M3 A and B, K-major, N = BR, M = BQ
  static constexpr uint32_t IDESC =
      (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(BR >> 3) << 17) | ((uint32_t)(BQ >> 4) << 24);
};
template <class F>
struct Tiles {
  static constexpr uint32_t BYTES = (uint32_t)BQ * F::ROW_BYTES;  // one 128-row operand tile
};
constexpr uint32_t BF_TILE = Tiles<FmtBF16>::BYTES;  // 28672
constexpr uint32_t F8_TILE = Tiles<FmtFP8>::BYTES;   // 16384

template <class F>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  if constexpr (F::kFP8) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(F::IDESC), "r"(accumulate));
  } else {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(F::IDESC), "r"(accumulate));
  }
}

// max of 32 values as a tree of three-input maxima (16 instructions)
__device__ __forceinline__ float max32(const float *v) {
  float a[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) a[k] = fmax3(v[3 * k], v[3 * k + 1], v[3 * k + 2]);
  const float b0 = fmax3(a[0], a[1], a[2]), b1 = fmax3(a[3], a[4], a[5]), b2 = fmax3(a[6], a[7], a[8]);
  const float b3 = fmax3(a[9], v[30], v[31]);
  return fmax3(b0, b1, fmaxf(b2, b3));
}

// bit j set iff v[j] >= t, built as four independent chains
__device__ __forceinline__ uint32_t ge_mask32(const float *v, float t) {
  uint32_t p[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int g = 0; g < 4; ++g) p[g] |= (v[g * 8 + j] >= t ? 1u : 0u) << (g * 8 + j);
  return (p[0] | p[1]) | (p[2] | p[3]);
}

// ------------------------------------------------------------- build ---

__global__ void k_build_bf16_blocks(const float *__restrict__ vecs, const float *__restrict__ norms,
                                    const uint32_t *__restrict__ perm, uint64_t n, __nv_bfloat16 *__restrict__ out) {
  const uint64_t b = blockIdx.x;
  constexpr int BK = FmtBF16::K;
  __nv_bfloat16 *o = out + b * (BF_TILE / 2);
  for (uint32_t i = threadIdx.x; i < (uint32_t)BR * BK; i += blockDim.x) {
    const uint32_t r = i / BK, k = i % BK;
    const uint64_t p = b * BR + r;
    float v = 0.f;
    if (p < n) {
      const uint32_t id = perm[p];
      if (k < (uint32_t)DIM) {
        v = vecs[(uint64_t)id * DIM + k];
      } else if (k == DIM || k == DIM + 1) {
        const float h = -0.5f * norms[id];
        const float hi = __bfloat162float(__float2bfloat16_rn(h));
        v = (k == DIM) ? hi : h - hi;
      }
    }
    o[cm_index(r, k)] = __float2bfloat16_rn(v);
  }
}

// Where a tile's lanes come from: the host plan's per-tile arrays, or a
// device plan's sorted queries (tile t = positions tile_first[t] ..
// + tiles[t].nq of order_q, slabs from the query descriptors).
struct LaneSrc {
  const int32_t *lane_q = nullptr;
  const uint32_t *lane_s = nullptr, *lane_e = nullptr;
  const uint32_t *tile_first = nullptr, *order_q = nullptr;
  const QueryDesc *desc = nullptr;
  const uint32_t *ntile = nullptr;  // device plan: the tile count
};

__device__ __forceinline__ int32_t lane_query(const LaneSrc &ls, const Tile &tl, uint32_t t, int L, uint32_t &s,
                                              uint32_t &e) {
  if (ls.lane_q) {
    const int32_t qi = ls.lane_q[t * BQ + L];
    if (qi >= 0) {
      s = ls.lane_s[t * BQ + L];
      e = ls.lane_e[t * BQ + L];
    }
    return qi;
  }
  if ((uint32_t)L >= tl.nq) return -1;
  const int32_t qi = (int32_t)ls.order_q[ls.tile_first[t] + L];
  s = ls.desc[qi].s;
  e = ls.desc[qi].e;
  return qi;
}

// One block per tile (grid-strided over a device plan's tile count).
__global__ void k_tile_stage_bf16(const float *__restrict__ q, LaneSrc ls, const Tile *__restrict__ tiles,
                                  uint32_t ntile_h, const QueryDesc *__restrict__ desc,
                                  __nv_bfloat16 *__restrict__ out, float2 *__restrict__ lane_qs) {
  constexpr int BK = FmtBF16::K;
  const uint32_t ntile = ls.ntile ? *ls.ntile : ntile_h;
  __shared__ int32_t lq[BQ];
  for (uint32_t t = blockIdx.x; t < ntile; t += gridDim.x) {
    const Tile tl = tiles[t];
    __nv_bfloat16 *o = out + (uint64_t)t * (BF_TILE / 2);
    for (uint32_t l = threadIdx.x; l < (uint32_t)BQ; l += blockDim.x) {
      uint32_t s_, e_;
      const int32_t qi = lane_query(ls, tl, t, (int)l, s_, e_);
      lq[l] = qi;
      lane_qs[t * BQ + l] = make_float2(qi >= 0 ? desc[qi].qn : 0.f, 1.f);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < (uint32_t)BQ * BK; i += blockDim.x) {
      const uint32_t l = i / BK, k = i % BK;
      const int32_t qi = lq[l];
      float v = 0.f;
      if (qi >= 0) {
        if (k < (uint32_t)DIM) v = q[(uint64_t)qi * DIM + k];
        else if (k == DIM || k == DIM + 1) v = 1.f;
      }
      o[cm_index(l, k)] = __float2bfloat16_rn(v);
    }
    __syncthreads();
  }
}

// FP8-e4m3 per-dimension-scaled codes, the tensor-core analogue of the
// per-dimension SQ8 codes of sq8_quant.hpp:30-63 (mi/dif per dimension).
// Each dimension is centred at c = (max + min)/2 and scaled by
// s = (max - min)/2 / 448 so its range fills e4m3 (|x'| <= 448):
//   row side : x'_k = e4m3((x_k - c_k) / s_k), k < 100; dims 100..102 hold
//              -|x - c|^2/2 as e4m3 high, middle and low parts
//   query    : A_k = e4m3(lambda * (q_k - c_k) * s_k); dims 100..102 = lambda,
//              lambda a power of two in [2^-9, 2^8] with max|A_k| <= 448
// so acc = lambda * ((q - c).(x - c) - |x - c|^2/2) and
// ds = |q - c|^2 - 2 acc / lambda approximates |q - x|^2.
__global__ void k_dim_minmax(const float *__restrict__ vecs, uint64_t n, uint32_t *__restrict__ mn,
                             uint32_t *__restrict__ mx) {
  __shared__ uint32_t smn[DIM], smx[DIM];
  for (int d = threadIdx.x; d < DIM; d += blockDim.x) {
    smn[d] = 0xffffffffu;
    smx[d] = 0u;
  }
  __syncthreads();
  const uint64_t total = n * DIM;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = f32_sortable(vecs[i]);
    const int d = (int)(i % DIM);
    atomicMin(&smn[d], u);
    atomicMax(&smx[d], u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < DIM; d += blockDim.x) {
    atomicMin(&mn[d], smn[d]);
    atomicMax(&mx[d], smx[d]);
  }
}

__global__ void k_fp8_params(const uint32_t *__restrict__ mn, const uint32_t *__restrict__ mx,
                             float *__restrict__ center, float *__restrict__ scale) {
  const int d = threadIdx.x;
  if (d >= DIM) return;
  const float a = sortable_f32(mn[d]), b = sortable_f32(mx[d]);
  center[d] = 0.5f * (a + b);
  scale[d] = fmaxf(0.5f * (b - a), 1e-30f) / 448.f;
}

__global__ void k_build_fp8_blocks(const float *__restrict__ vecs, const uint32_t *__restrict__ perm, uint64_t n,
                                   const float *__restrict__ center, const float *__restrict__ scale,
                                   unsigned char *__restrict__ out) {
  const uint64_t b = blockIdx.x;
  unsigned char *o = out + b * F8_TILE;
  __shared__ float cn[BR];
  // centred norms of the block's rows (float FMA chain)
  for (uint32_t r = threadIdx.x; r < (uint32_t)BR; r += blockDim.x) {
    const uint64_t p = b * BR + r;
    float s = 0.f;
    if (p < n) {
      const float *x = vecs + (uint64_t)perm[p] * DIM;
      for (int k = 0; k < DIM; ++k) {
        const float t = x[k] - center[k];
        s = fmaf(t, t, s);
      }
    }
    cn[r] = s;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < (uint32_t)BR * FmtFP8::K; i += blockDim.x) {
    const uint32_t r = i / FmtFP8::K, k = i % FmtFP8::K;
    const uint64_t p = b * BR + r;
    float v = 0.f;
    if (p < n) {
      if (k < (uint32_t)DIM) {
        v = (vecs[(uint64_t)perm[p] * DIM + k] - center[k]) / scale[k];
      } else if (k <= DIM + 2) {
        const float h = -0.5f * cn[r];
        const float hi = float(__nv_fp8_e4m3(h));
        const float mid = float(__nv_fp8_e4m3(h - hi));
        v = (k == DIM) ? hi : (k == DIM + 1) ? mid : h - hi - mid;
      }
    }
    o[cm_byte(r, k)] = __nv_fp8_e4m3(v).__x;
  }
}

__global__ void k_tile_stage_fp8(const float *__restrict__ q, LaneSrc ls, const Tile *__restrict__ tiles,
                                 uint32_t ntile_h, const float *__restrict__ center, const float *__restrict__ scale,
                                 unsigned char *__restrict__ out, float2 *__restrict__ lane_qs) {
  const uint32_t ntile = ls.ntile ? *ls.ntile : ntile_h;
  __shared__ float lam[BQ];
  __shared__ int32_t lq[BQ];
  for (uint32_t t = blockIdx.x; t < ntile; t += gridDim.x) {
    const Tile tl = tiles[t];
    unsigned char *o = out + (uint64_t)t * F8_TILE;
    for (uint32_t l = threadIdx.x; l < (uint32_t)BQ; l += blockDim.x) {
      uint32_t s_, e_;
      const int32_t qi = lane_query(ls, tl, t, (int)l, s_, e_);
      lq[l] = qi;
      float qn = 0.f, mw = 0.f;
      if (qi >= 0) {
        const float *x = q + (uint64_t)qi * DIM;
        for (int k = 0; k < DIM; ++k) {
          const float u = x[k] - center[k];
          qn = fmaf(u, u, qn);
          mw = fmaxf(mw, fabsf(u * scale[k]));
        }
      }
      // largest power of two with lambda * max|w| <= 448, within e4m3's exact powers
      int e = 8;
      if (mw > 0.f) e = min(8, max(-9, (int)floorf(log2f(448.f / mw))));
      const float lambda = ldexpf(1.f, e);
      lam[l] = lambda;
      lane_qs[t * BQ + l] = make_float2(qn, 1.f / lambda);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < (uint32_t)BQ * FmtFP8::K; i += blockDim.x) {
      const uint32_t l = i / FmtFP8::K, k = i % FmtFP8::K;
      const int32_t qi = lq[l];
      float v = 0.f;
      if (qi >= 0) {
        if (k < (uint32_t)DIM) v = lam[l] * (q[(uint64_t)qi * DIM + k] - center[k]) * scale[k];
        else if (k <= DIM + 2) v = lam[l];
      }
      o[cm_byte(l, k)] = __nv_fp8_e4m3(v).__x;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ screen ---

template <class F>
struct BScreenSmem {
  unsigned char a[Tiles<F>::BYTES];
  unsigned char b[BS][Tiles<F>::BYTES];
  float thr[BQ];  // current k'-th screening distance bound T
  float qn[BQ];
  int cnt[BQ];
  int32_t lq[BQ];
  uint32_t hist[B_EPI_WARPS][256];
  // per epilogue lane, the 32 accumulator columns of a chunk that has
  // candidates (rows padded to 36 floats: conflict-free 16-byte stores)
  float stage[B_EPI_WARPS][32 * STAGE_ROW];
  uint64_t full[BS], empty[BS], accfull[2], accempty[2], abar;
  uint32_t tmem_base;
  uint32_t next[2];  // the next processing slot, by item parity (work queue)
};

// two screening CTAs share an SM (228 KB of shared memory, 1 KB reserved per CTA)
static_assert(sizeof(BScreenSmem<FmtBF16>) <= 113 * 1024 && sizeof(BScreenSmem<FmtFP8>) <= 113 * 1024,
              "screen shared memory must leave room for two CTAs per SM");

// Screens 32 accumulator columns c .. c+31 of one query (this lane): every
// column j inside the slab [r0, r1) with acc >= cq is appended to the
// query's list with its screening distance qn - 2 sc acc.  The lane's
// candidates form a bit mask; their values are read back from the lane's
// shared-memory staging row, so the push loop runs once per candidate.
__device__ __forceinline__ int screen_chunk(const uint32_t (&r)[32], int c, int r0, int r1, float cq, float qn,
                                            float sc, uint32_t p0, float *row, Candidate *list, int cnt) {
  if (r0 >= c + 32 || r1 <= c) return cnt;
  float v[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
  if (!(r0 <= c && r1 >= c + 32)) {
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (c + j < r0 || c + j >= r1) v[j] = -INFINITY;
  }
  if (max32(v) >= cq) {
    uint32_t mask = ge_mask32(v, cq);
#pragma unroll
    for (int j = 0; j < 32; j += 4)
      *reinterpret_cast<float4 *>(row + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
    while (mask) {
      const int j = __ffs(mask) - 1;
      mask &= mask - 1;
      Candidate cd;
      cd.ds = fmaf(-2.f * sc, row[j], qn);
      cd.pos = p0 + c + j;
      list[cnt++] = cd;
    }
  }
  return cnt;
}

// kth smallest (1-based) of the n keys held NPL per lane (element
// j*32 + lane in key[j]; keys past n ignored): a warp radix select that
// starts below the bits all keys share and takes up to 8 bits per pass from
// a shared-memory histogram.  Keys are order-preserving images of floats.
template <int NPL>
__device__ __forceinline__ uint32_t warp_kth_regs(const uint32_t (&key)[NPL], int n, int kth, uint32_t *hist) {
  const int lane = threadIdx.x & 31;
  uint32_t mn = 0xffffffffu, mx = 0u;
#pragma unroll
  for (int j = 0; j < NPL; ++j)
    if (j * 32 + lane < n) {
      mn = min(mn, key[j]);
      mx = max(mx, key[j]);
    }
  mn = __reduce_min_sync(0xffffffffu, mn);
  mx = __reduce_max_sync(0xffffffffu, mx);
  if (mn == mx) return mn;
  int hi = 32 - __clz(mn ^ mx);  // bits [hi-1, 0] still differ
  uint32_t mask = hi == 32 ? 0u : ~((1u << hi) - 1u);
  uint32_t prefix = mn & mask;
  int remaining = kth;
  while (hi > 0) {
    const int w = min(8, hi), shift = hi - w;
    const uint32_t nb = 1u << w;
    for (uint32_t i = lane; i < 256; i += 32) hist[i] = 0;
    __syncwarp();
#pragma unroll
    for (int j = 0; j < NPL; ++j)
      if (j * 32 + lane < n && (key[j] & mask) == prefix) atomicAdd(&hist[(key[j] >> shift) & (nb - 1)], 1u);
    __syncwarp();
    uint32_t local[8], sum = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      local[j] = hist[lane * 8 + j];
      sum += local[j];
    }
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += v;
    }
    const uint32_t excl = inc - sum;
    const uint32_t hit = __ballot_sync(0xffffffffu, excl < (uint32_t)remaining && inc >= (uint32_t)remaining);
    const int owner = __ffs(hit) - 1;
    uint32_t bin = 0, before = 0;
    if (lane == owner) {
      uint32_t c = excl;
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (c + local[j] >= (uint32_t)remaining) {
          bin = lane * 8 + j;
          before = c;
          break;
        } else {
          c += local[j];
        }
    }
    bin = __shfl_sync(0xffffffffu, bin, owner);
    before = __shfl_sync(0xffffffffu, before, owner);
    remaining -= (int)before;
    prefix |= bin << shift;
    mask |= (nb - 1) << shift;
    hi = shift;
    __syncwarp();
  }
  return prefix;
}

// Bound and trim list L to its k' smallest screening distances (ties kept):
// the list (n <= 32 * NPL entries) is read once into registers, its k'-th
// key selected there, the bound shared through T_global, and the kept
// entries written back in order.
template <class F, int NPL>
__device__ __noinline__ void bcompact(Candidate *list, BScreenSmem<F> &sm, int L, int wslot, uint32_t kprime,
                                      uint32_t capb, uint32_t *T_global, uint32_t *ovf) {
  const int lane = threadIdx.x & 31;
  const int n = sm.cnt[L];
  const int32_t qi = sm.lq[L];
  float T = sm.thr[L];
  uint32_t key[NPL], pos[NPL];
  const uint2 *src = reinterpret_cast<const uint2 *>(list);
#pragma unroll
  for (int j = 0; j < NPL; ++j) {
    const int i = j * 32 + lane;
    uint2 c = make_uint2(0xffffffffu, 0u);
    if (i < n) c = src[i];
    key[j] = i < n ? f32_sortable(__uint_as_float(c.x)) : 0xffffffffu;
    pos[j] = c.y;
  }
  if (n >= (int)kprime) T = fminf(T, sortable_f32(warp_kth_regs<NPL>(key, n, (int)kprime, sm.hist[wslot])));
  const float Tg = sortable_f32(ld_volatile_u32(T_global + qi));
  if (Tg < T) T = Tg;
  if (lane == 0 && T < Tg) atomicMin(T_global + qi, f32_sortable(T));
  const uint32_t tk = f32_sortable(T);
  int kept = 0;
  const uint32_t lt = (1u << lane) - 1u;
  uint2 *dst = reinterpret_cast<uint2 *>(list);
  __syncwarp();
#pragma unroll
  for (int j = 0; j < NPL; ++j) {
    const bool keep = j * 32 + lane < n && key[j] <= tk;
    const uint32_t b = __ballot_sync(0xffffffffu, keep);
    if (keep) dst[kept + __popc(b & lt)] = make_uint2(__float_as_uint(sortable_f32(key[j])), pos[j]);
    kept += __popc(b);
  }
  __syncwarp();
  if (lane == 0) {
    if (kept > (int)capb - BR) {
      ovf[qi] = 1u;  // a tie flood: the exact scan answers this query
      sm.cnt[L] = 0;
      sm.thr[L] = -INFINITY;
    } else {
      sm.cnt[L] = kept;
      sm.thr[L] = T;
    }
  }
  __syncwarp();
}

// One CTA per resident slot; it works through the items blockIdx.x,
// blockIdx.x + gridDim.x, ... (a host plan launches one CTA per item, a
// device plan a fixed grid over the device item count).  The barrier
// phases run on across items: g counts the sub-tiles this CTA has issued.
template <class F, int NPL>
__global__ void __launch_bounds__(B_THREADS, 2)
    k_screen_tc(const WorkItem *__restrict__ items, const Tile *__restrict__ tiles,
                const unsigned char *__restrict__ atiles, LaneSrc ls, const float2 *__restrict__ lane_qs,
                const unsigned char *__restrict__ blocks_t, const unsigned char *__restrict__ blocks_c,
                uint32_t *__restrict__ T_global, uint32_t *__restrict__ ovf, Candidate *__restrict__ out,
                uint32_t *__restrict__ out_cnt, uint32_t kprime, uint32_t capb, uint32_t refresh, uint32_t stride,
                uint32_t withhold, uint32_t nitems_h, const uint32_t *__restrict__ nitems_d,
                const uint32_t *__restrict__ order, uint32_t *queue, int *err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  BScreenSmem<F> &sm = *reinterpret_cast<BScreenSmem<F> *>(smem_raw);
  constexpr uint32_t TB = Tiles<F>::BYTES;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t nitems = nitems_d ? *nitems_d : nitems_h;
  if (blockIdx.x >= nitems) return;  // (uniform: before any barrier or TMEM use)

  if (tid == 0) {
    for (int s = 0; s < BS; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&sm.accfull[a], 1);
      mbar_init(&sm.accempty[a], B_EPI_WARPS);
    }
    mbar_init(&sm.abar, 1);
    fence_mbar_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  uint32_t g = 0;  // sub-tiles of this CTA's earlier items
  uint32_t iter = 0;
  // a bounded wait gave up: the CTA's later items only mark their queries
  // (combined over the block at each item's closing barrier, so uniform)
  bool aborted = false;
  // processing slots: blockIdx.x first, then the next free slot of the work
  // queue (queue != NULL) or blockIdx.x + k * gridDim.x; slot -> item
  // through order (longest first) when given
  for (uint32_t slot = blockIdx.x; slot < nitems; ++iter) {
    const uint32_t item_id = order ? order[slot] : slot;
    const WorkItem it = items[item_id];
    const Tile tl = tiles[it.tile];
    const unsigned char *blocks = tl.order == ORDER_TIME ? blocks_t : blocks_c;
    // every stride-th row block of the item (stride 1: all of them)
    const uint32_t nsub = (it.blk1 - it.blk0 + stride - 1) / stride;
    bool gave_up = false;  // this thread saw a wait give up in this item

    if (warp == 0) {
      // ------------------------------------------------ producer
      if (lane == 0 && !aborted) {
        bool ok = true;
        mbar_arrive_expect_tx(&sm.abar, TB);
        bulk_g2s(sm.a, atiles + (uint64_t)it.tile * TB, TB, &sm.abar);
        uint32_t issued = 0;
        // test hook (fknn_index_test_withhold_copy): the first work item issues
        // no row-block copy, so its MMA issuer's and epilogue's waits run out
        const uint32_t nsub_issue = (withhold && item_id == 0) ? 0u : nsub;
        for (uint32_t sub = 0; sub < nsub_issue; ++sub) {
          const uint32_t gs = g + sub;
          const int st = gs % BS;
          if (gs >= BS && !mbar_wait_bounded(&sm.empty[st], ((gs / BS) - 1) & 1, err)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&sm.full[st], TB);
          bulk_g2s(sm.b[st], blocks + (uint64_t)(it.blk0 + sub * stride) * TB, TB, &sm.full[st]);
          ++issued;
        }
        // every issued copy has landed before the item ends
        ok = mbar_wait_bounded(&sm.abar, iter & 1, err) && ok;
        for (uint32_t i = issued > BS ? issued - BS : 0; i < issued; ++i)
          ok = mbar_wait_bounded(&sm.full[(g + i) % BS], ((g + i) / BS) & 1, err) && ok;
        if (!ok || issued != nsub) gave_up = true;
      }
    } else if (warp == 1) {
      // ------------------------------------------------ MMA issuer
      if (lane == 0 && !aborted) {
        uint32_t done = 0;
        if (mbar_wait_bounded(&sm.abar, iter & 1, err)) {
          const uint32_t a0 = smem_u32(sm.a);
          for (uint32_t sub = 0; sub < nsub; ++sub) {
            const uint32_t gs = g + sub;
            const int st = gs % BS, ab = gs & 1;
            if (!mbar_wait_bounded(&sm.full[st], (gs / BS) & 1, err)) break;
            if (gs >= 2 && !mbar_wait_bounded(&sm.accempty[ab], ((gs >> 1) - 1) & 1, err)) break;
            tc_fence_after();
            const uint32_t b0 = smem_u32(sm.b[st]);
#pragma unroll
            for (int kk = 0; kk < F::MMAS; ++kk) {
              const uint64_t da = umma_desc(a0 + kk * 2 * (BQ / 8) * 128, (BQ / 8) * 128, 128);
              const uint64_t db = umma_desc(b0 + kk * 2 * (BR / 8) * 128, (BR / 8) * 128, 128);
              umma<F>(tmem + ab * BR, da, db, kk > 0);
            }
            umma_commit(&sm.empty[st]);     // the row block may be overwritten once these MMAs finish
            umma_commit(&sm.accfull[ab]);   // the accumulator is ready for the epilogue
            ++done;
          }
        }
        // no MMA of this item is in flight when the next item (or the dealloc) comes
        if (done) {
          const uint32_t gl = g + done - 1;
          mbar_wait_bounded(&sm.accfull[gl & 1], (gl >> 1) & 1, err);
        }
        if (done != nsub) gave_up = true;
      }
    } else {
      // ------------------------------------------------ epilogue: thread = query
      const int wslot = warp - 2;
      const int wg = warp & 3;  // TMEM lanes 32*wg .. 32*wg+31 are reachable from this warp
      const int L = wg * 32 + lane;
      uint32_t s = 0, e = 0;
      const int32_t qi = lane_query(ls, tl, it.tile, L, s, e);
      // per query: |q|^2 (centred for FP8) and the accumulator's scale 1/lambda
      const float2 qsc = lane_qs[it.tile * BQ + L];
      const float qn = qsc.x, sc = qsc.y;
      float T = -INFINITY;
      if (qi >= 0) {
        T = sortable_f32(ld_volatile_u32(T_global + qi));
        if (ld_volatile_u32(ovf + qi)) T = -INFINITY;
      }
      sm.lq[L] = qi;
      sm.cnt[L] = 0;
      sm.thr[L] = T;
      __syncwarp();
      Candidate *list = out + ((uint64_t)item_id * BQ + L) * capb;
      int cnt = 0;
      bool ok = !aborted;
      // candidate iff qn - 2*sc*acc <= T  <=>  acc >= (qn - T) / (2 sc);
      // with no bound yet every column of the slab is one (cq = -FLT_MAX),
      // and columns outside the slab are -inf, which no cq admits.  cq is
      // recomputed only when T changes.
      auto acc_bound = [&](float t) { return (t == INFINITY) ? -FLT_MAX : 0.5f * (qn - t) / sc; };
      float cq = acc_bound(T);
      uint32_t until_refresh = refresh;  // sub-tiles until the next read of the shared bound
      for (uint32_t sub = 0; sub < nsub && ok; ++sub) {
        const uint32_t gs = g + sub;
        const int ab = gs & 1;
        // warp-uniform: the lanes' timers may disagree at the deadline
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&sm.accfull[ab], (gs >> 1) & 1, err))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t p0 = (it.blk0 + sub * stride) * BR;
        const int r0 = (int)min(max(s, p0), p0 + BR) - (int)p0;
        const int r1 = (int)min(max(e, p0), p0 + BR) - (int)p0;
        // four 32-column chunks; the TMEM load of the next chunk is in flight
        // while this one is screened
        const uint32_t tb = tmem + ((uint32_t)(wg * 32) << 16) + ab * BR;
        uint32_t ra[32], rb[32];
        tmem_ld32_issue(tb, ra);
        tmem_wait_ld(ra);
        tmem_ld32_issue(tb + 32, rb);
        cnt = screen_chunk(ra, 0, r0, r1, cq, qn, sc, p0, &sm.stage[wslot][lane * STAGE_ROW], list, cnt);
        __syncwarp();
        tmem_wait_ld(rb);
        tmem_ld32_issue(tb + 64, ra);
        cnt = screen_chunk(rb, 32, r0, r1, cq, qn, sc, p0, &sm.stage[wslot][lane * STAGE_ROW], list, cnt);
        __syncwarp();
        tmem_wait_ld(ra);
        tmem_ld32_issue(tb + 96, rb);
        cnt = screen_chunk(ra, 64, r0, r1, cq, qn, sc, p0, &sm.stage[wslot][lane * STAGE_ROW], list, cnt);
        __syncwarp();
        tmem_wait_ld(rb);
        cnt = screen_chunk(rb, 96, r0, r1, cq, qn, sc, p0, &sm.stage[wslot][lane * STAGE_ROW], list, cnt);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive1(&sm.accempty[ab]);
        // lists that could overflow in the next sub-tile are bounded and
        // trimmed; counts and bounds pass through shared memory only then
        uint32_t msk = __ballot_sync(0xffffffffu, cnt > (int)capb - BR);
        if (msk) {
          sm.cnt[L] = cnt;
          __syncwarp();
          while (msk) {
            const int b = __ffs(msk) - 1;
            msk &= msk - 1;
            const int Lb = wg * 32 + b;
            bcompact<F, NPL>(out + ((uint64_t)item_id * BQ + Lb) * capb, sm, Lb, wslot, kprime, capb, T_global, ovf);
          }
          cnt = sm.cnt[L];
          T = sm.thr[L];
          cq = acc_bound(T);
        }
        // other items of the same query tighten the shared bound meanwhile
        // (every refresh-th sub-tile of the item)
        if (refresh && --until_refresh == 0) {
          until_refresh = refresh;
          if (qi >= 0) {
            const float Tg = sortable_f32(ld_volatile_u32(T_global + qi));
            if (Tg < T) {
              T = Tg;
              sm.thr[L] = T;
              cq = acc_bound(T);
            }
          }
        }
      }
      if (!ok) {
        // this item's queries are answered by the exact scan
        if (qi >= 0) ovf[qi] = 1u;
        out_cnt[(uint64_t)item_id * BQ + L] = 0;
        gave_up = true;
      } else {
        sm.cnt[L] = cnt;
        __syncwarp();
        for (int b = 0; b < 32; ++b) {
          const int Lb = wg * 32 + b;
          if (sm.cnt[Lb] > 0 && sm.lq[Lb] >= 0)
            bcompact<F, NPL>(out + ((uint64_t)item_id * BQ + Lb) * capb, sm, Lb, wslot, kprime, capb, T_global,
                             ovf);
        }
        out_cnt[(uint64_t)item_id * BQ + L] = (uint32_t)sm.cnt[L];
      }
    }
    g += nsub;
    // double-buffered by item parity: a slow thread may still read the slot
    // of this barrier while thread 0 writes the one after
    if (queue && tid == 0) sm.next[(iter + 1) & 1] = atomicAdd(queue, 1u) + gridDim.x;
    tc_fence_before();
    // the item's shared state (A tile, lists' counts, bounds) is reused by the next
    aborted = __syncthreads_or(aborted || gave_up) != 0;
    tc_fence_after();
    slot = queue ? sm.next[(iter + 1) & 1] : slot + gridDim.x;
  }
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// ------------------------------------------------------------ re-rank --

constexpr int RR_THREADS = 256;
constexpr int RR_CAP = 8192;        // screening candidates the large merge holds
constexpr int RR_CAP_SMALL = 2048;  // ... and the common one (8 blocks per SM)
constexpr int RR_KMAX = 1024;       // largest k'

template <int CAP>
struct RerankSmem {
  float key[CAP];
  uint32_t val[CAP];
  uint64_t ekey[RR_KMAX];
  float qv[DIM];
  uint32_t cnt_prefix[RR_THREADS + 1];
  int total;
};

struct MergeArgs {
  const uint32_t *big_q, *big_tile, *big_lane;
  const Tile *tiles;
  const uint32_t *item_slot;
  const Candidate *out;
  const uint32_t *out_cnt;
  const QueryDesc *desc;
  const float *q, *vecs;
  const uint32_t *perm_t, *perm_c, *ovf;
  uint32_t *ovf_list, *ovf_count;
  uint32_t k, kprime, capb;
  const uint32_t *seeded;
  uint32_t *ids;
  float *dists;
  uint32_t *n_f64;
  const uint32_t *nbig_d;  // device plan: the big-query count (NULL: the launch's nbig)
};

// One big query b (index into the plan's big-query arrays): gather its
// lists, keep the k' best screening distances, re-rank them in FP32.  A
// query with more than CAP candidates goes to `spill` (the large merge) or,
// from the large merge, to the exact scan.  Returns are block-uniform.
template <int CAP>
__device__ void merge_one(const MergeArgs &A, uint32_t b, RerankSmem<CAP> &sm, uint32_t *spill,
                          uint32_t *spill_count) {
  const uint32_t *big_tile = A.big_tile, *big_lane = A.big_lane, *item_slot = A.item_slot, *out_cnt = A.out_cnt;
  const Tile *tiles = A.tiles;
  const Candidate *out = A.out;
  const QueryDesc *desc = A.desc;
  const float *q = A.q, *vecs = A.vecs;
  const uint32_t *perm_t = A.perm_t, *perm_c = A.perm_c, *seeded = A.seeded;
  uint32_t *ovf_list = A.ovf_list, *ovf_count = A.ovf_count, *ids = A.ids, *n_f64 = A.n_f64;
  float *dists = A.dists;
  const uint32_t k = A.k, kprime = A.kprime, capb = A.capb;
  const int tid = threadIdx.x;
  const uint32_t qi = A.big_q[b];
  if (A.ovf[qi]) {
    if (tid == 0) ovf_list[atomicAdd(ovf_count, 1u)] = qi;
    return;
  }
  const Tile tl = tiles[big_tile[b]];
  const uint32_t L = big_lane[b];
  const uint32_t nitems = tl.item1 - tl.item0;
  const QueryDesc dsc = desc[qi];
  for (int d = tid; d < DIM; d += RR_THREADS) sm.qv[d] = q[(uint64_t)qi * DIM + d];
  // candidate counts of the query's items (a tile has at most a few dozen)
  // more items than prefix slots: the exact scan answers the query
  list_offsets(item_slot, tl.item0, nitems, out_cnt, L, BQ, sm.cnt_prefix, &sm.total, RR_THREADS, RR_CAP + 1);
  __syncthreads();
  const int M = sm.total;
  if (M > CAP && spill && M <= RR_CAP) {  // the large merge takes it
    if (tid == 0) spill[atomicAdd(spill_count, 1u)] = b;
    return;
  }
  // a pilot bound that kept fewer than k' rows was set too low: the exact
  // scan answers the query
  if (M > CAP || (seeded && seeded[qi] && M < (int)kprime)) {
    if (tid == 0) ovf_list[atomicAdd(ovf_count, 1u)] = qi;
    return;
  }
  // the whole block copies each item's list
  for (uint32_t i = 0; i < nitems; ++i) {
    const uint64_t item = item_slot ? item_slot[tl.item0 + i] : tl.item0 + i;
    const uint32_t base = sm.cnt_prefix[i];
    const uint32_t c = (i + 1 < nitems ? sm.cnt_prefix[i + 1] : (uint32_t)M) - base;
    const Candidate *src = out + (item * BQ + L) * capb;
    for (uint32_t j = tid; j < c; j += RR_THREADS) {
      const Candidate cd = src[j];
      sm.key[base + j] = cd.ds;
      sm.val[base + j] = cd.pos;
    }
  }
  int np2 = 32;
  while (np2 < M) np2 <<= 1;
  for (int i = M + tid; i < np2; i += RR_THREADS) {
    sm.key[i] = INFINITY;
    sm.val[i] = 0xffffffffu;
  }
  __syncthreads();
  block_bitonic_sort_kv(sm.key, sm.val, np2);
  // FP32 re-rank of the k' best screened rows with the reference's arithmetic
  const int C = min(M, (int)kprime);
  const uint32_t *perm = dsc.order == ORDER_TIME ? perm_t : perm_c;
  for (int i = tid; i < C; i += RR_THREADS) {
    const uint32_t id = perm[sm.val[i]];
    const float d = seq_l2_strided(vecs + (uint64_t)id * DIM, 1, sm.qv);
    sm.ekey[i] = exact_key(d, id);
  }
  int cp2 = 32;
  while (cp2 < C) cp2 <<= 1;
  for (int i = C + tid; i < cp2; i += RR_THREADS) sm.ekey[i] = ~0ull;
  __syncthreads();
  block_bitonic_sort(sm.ekey, cp2);
  // FP64 at the k-th boundary: candidates within 1e-6 relative of the k-th
  // FP32 distance are ordered by their exact double distance
  if (tid == 0 && C > 0) {
    const int kk = min((int)k, C);
    const float D = sortable_f32((uint32_t)(sm.ekey[kk - 1] >> 32));
    const float lo = D - 1e-6f * D, hi = D + 1e-6f * D;
    int i0 = kk - 1, i1 = kk;
    while (i0 > 0 && sortable_f32((uint32_t)(sm.ekey[i0 - 1] >> 32)) >= lo) --i0;
    while (i1 < C && sortable_f32((uint32_t)(sm.ekey[i1] >> 32)) <= hi) ++i1;
    if (i1 - i0 > 1) {
      double d64[64];
      const int nb = min(i1 - i0, 64);
      for (int j = 0; j < nb; ++j) {
        const uint32_t id = (uint32_t)sm.ekey[i0 + j];
        const float *x = vecs + (uint64_t)id * DIM;
        double s = 0.0;
        for (int d = 0; d < DIM; ++d) {
          const double t = (double)x[d] - (double)sm.qv[d];
          s += t * t;
        }
        d64[j] = s;
      }
      for (int a = 1; a < nb; ++a) {  // insertion sort by (d64, id)
        const double dv = d64[a];
        const uint64_t kv = sm.ekey[i0 + a];
        int b = a - 1;
        while (b >= 0 && (d64[b] > dv || (d64[b] == dv && (uint32_t)sm.ekey[i0 + b] > (uint32_t)kv))) {
          d64[b + 1] = d64[b];
          sm.ekey[i0 + b + 1] = sm.ekey[i0 + b];
          --b;
        }
        d64[b + 1] = dv;
        sm.ekey[i0 + b + 1] = kv;
      }
      atomicAdd(n_f64, (uint32_t)nb);
    }
  }
  __syncthreads();
  for (uint32_t j = tid; j < k; j += RR_THREADS) {
    uint32_t id = 0xffffffffu;
    float d = INFINITY;
    if ((int)j < C) {
      id = (uint32_t)sm.ekey[j];
      d = sortable_f32((uint32_t)(sm.ekey[j] >> 32));
    }
    ids[(uint64_t)qi * k + j] = id;
    if (dists) dists[(uint64_t)qi * k + j] = d;
  }
}

// work == nullptr: block b merges big query b (grid = number of big
// queries); else the blocks stride over the *work_count entries of work.
template <int CAP>
__global__ void __launch_bounds__(RR_THREADS)
    k_merge_rerank(MergeArgs A, uint32_t nbig, const uint32_t *__restrict__ work,
                   const uint32_t *__restrict__ work_count, uint32_t *__restrict__ spill,
                   uint32_t *__restrict__ spill_count) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  RerankSmem<CAP> &sm = *reinterpret_cast<RerankSmem<CAP> *>(smem_raw);
  const uint32_t nwork = work ? *work_count : (A.nbig_d ? *A.nbig_d : nbig);
  for (uint32_t w = blockIdx.x; w < nwork; w += gridDim.x) {
    merge_one<CAP>(A, work ? work[w] : w, sm, spill, spill_count);
    __syncthreads();  // shared memory is reused by the next query
  }
}

// Seeds the shared bound of every long query from the pilot pass: T_A is
// the r-th smallest screening distance over every stride-th row block, an
// estimate of the k'-th over all rows (r is chosen so that it lies above it
// with high probability; the merge catches the rest).
__global__ void k_seed_bounds(const uint32_t *__restrict__ big_q, uint32_t nbig_h, const uint32_t *__restrict__ nbig_d,
                              const QueryDesc *__restrict__ desc, const uint32_t *__restrict__ T_A,
                              const uint32_t *__restrict__ ovf_A, uint32_t min_rows, uint32_t *__restrict__ T_global,
                              uint32_t *__restrict__ seeded) {
  const uint32_t nbig = nbig_d ? *nbig_d : nbig_h;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nbig; i += gridDim.x * blockDim.x) {
    const uint32_t qi = big_q[i];
    const uint32_t inf = f32_sortable(INFINITY);
    const bool s = desc[qi].e - desc[qi].s >= min_rows && T_A[qi] < inf && !ovf_A[qi];
    T_global[qi] = s ? T_A[qi] : inf;
    seeded[qi] = s ? 1u : 0u;
  }
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

int build_bf16(fknn_index *idx, cudaStream_t st) {
  const uint64_t nblk = (idx->n + BR - 1) / BR;
  for (int o = 0; o < 2; ++o) {
    int rc = dev_alloc(idx, &idx->bf16_blocks[o], nblk * BF_TILE);
    if (rc) return rc;
    k_build_bf16_blocks<<<(unsigned)nblk, 256, 0, st>>>(idx->vecs, idx->norms, idx->ord[o].perm, idx->n,
                                                        (__nv_bfloat16 *)idx->bf16_blocks[o]);
    g_launches += 1;
  }
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

int build_fp8(fknn_index *idx, cudaStream_t st) {
  const uint64_t nblk = (idx->n + BR - 1) / BR;
  int rc = dev_alloc(idx, (void **)&idx->fp8_scale, 2 * DIM * sizeof(float));  // centre[100], scale[100]
  if (rc) return rc;
  uint32_t *mm;
  if ((rc = ws_get(idx, 15, 2 * DIM * sizeof(uint32_t), (void **)&mm))) return rc;
  FKNN_CUDA(cudaMemsetAsync(mm, 0xff, DIM * sizeof(uint32_t), st));
  FKNN_CUDA(cudaMemsetAsync(mm + DIM, 0, DIM * sizeof(uint32_t), st));
  k_dim_minmax<<<148 * 4, 256, 0, st>>>(idx->vecs, idx->n, mm, mm + DIM);
  k_fp8_params<<<1, 128, 0, st>>>(mm, mm + DIM, idx->fp8_scale, idx->fp8_scale + DIM);
  g_launches += 2;
  for (int o = 0; o < 2; ++o) {
    if ((rc = dev_alloc(idx, &idx->fp8_blocks[o], nblk * F8_TILE))) return rc;
    k_build_fp8_blocks<<<(unsigned)nblk, 256, 0, st>>>(idx->vecs, idx->ord[o].perm, idx->n, idx->fp8_scale,
                                                       idx->fp8_scale + DIM, (unsigned char *)idx->fp8_blocks[o]);
    g_launches += 1;
  }
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

template <class F>
static int search_tc(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k, uint32_t kprime,
                     uint32_t *d_ids, float *d_dists, cudaStream_t st, fknn_search_stats *stats) {
  const uint64_t n = idx->n;
  constexpr uint32_t TB = Tiles<F>::BYTES;
  int rc;
  QueryDesc *d_desc, *h_desc;
  float *h_meta;
  if ((rc = prepare_queries(idx, d_q, d_meta, nq, st, &d_desc, &h_desc, &h_meta))) return rc;
  uint32_t nsmall_early = 0;
  if ((rc = launch_small_scans(idx, h_desc, d_desc, nq, d_q, k, d_ids, d_dists, st, &nsmall_early))) return rc;
  const fknn_tuning tune = idx->tuning[F::kFP8 ? FKNN_MODE_FP8_RERANK : FKNN_MODE_BF16_RERANK];
  // candidate slots per (item, query): k' plus the pushes between trims; a
  // list holds at most 1280 (32 lanes x 40 registers in the trim)
  const uint32_t capb =
      (uint32_t)std::min<size_t>(1280, align_up(kprime + std::max<uint32_t>(tune.list_slack, 2 * BR), 128));
  auto t0 = std::chrono::steady_clock::now();
  Plan &P = idx->plan;
  PlanShape shape;
  shape.tq = BQ;
  shape.blk_rows = BR;
  shape.small_slab = SMALL_SLAB;
  // candidate scratch (items x 128 x capb x 8 B) stays within ~8 GB
  const uint64_t per_item = (uint64_t)BQ * capb * sizeof(Candidate);
  const uint64_t tiles_est = std::max<uint64_t>(1, (nq + BQ - 1) / BQ);
  shape.max_items_per_tile = (uint32_t)std::max<uint64_t>(
      1, std::min<uint64_t>(RR_CAP / capb, (8ull << 30) / (per_item * tiles_est)));
  shape.min_chunk_blocks = tune.min_chunk_blocks;
  shape.target_items = idx->num_sms * tune.items_per_sm;
  make_plan(h_desc, h_meta, nq, n, shape, P);
  auto t1 = std::chrono::steady_clock::now();
  const uint32_t ntile = (uint32_t)P.tiles.size(), nitems = (uint32_t)P.items.size();
  const uint32_t nbig = (uint32_t)P.big.size(), nsmall = (uint32_t)P.small.size();
  std::vector<uint32_t> &slot = P.w_slot;
  slot.resize(nitems);
  {
    std::vector<uint32_t> &fill = P.w_fill;
    fill.resize(ntile);
    for (uint32_t t = 0; t < ntile; ++t) fill[t] = P.tiles[t].item0;
    for (uint32_t s = 0; s < nitems; ++s) slot[fill[P.items[s].tile]++] = s;
  }
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = align_up(off + bytes, 256);
    return o;
  };
  const size_t o_small = take(nsmall * 4), o_big = take(nbig * 4), o_btile = take(nbig * 4),
               o_blane = take(nbig * 4), o_tiles = take(ntile * sizeof(Tile)),
               o_items = take(nitems * sizeof(WorkItem)), o_lq = take((size_t)ntile * BQ * 4),
               o_ls = take((size_t)ntile * BQ * 4), o_le = take((size_t)ntile * BQ * 4), o_slot = take(nitems * 4);
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
  put(o_lq, P.lane_q.data(), (size_t)ntile * BQ * 4);
  put(o_ls, P.lane_s.data(), (size_t)ntile * BQ * 4);
  put(o_le, P.lane_e.data(), (size_t)ntile * BQ * 4);
  put(o_slot, slot.data(), nitems * 4);
  if (blob) FKNN_CUDA(cudaMemcpyAsync(d_blob, h_blob, blob, cudaMemcpyHostToDevice, st));
  uint32_t *d_state;
  if ((rc = ws_get(idx, 5, (size_t)nq * 16 + 64, (void **)&d_state))) return rc;
  uint32_t *T_global = d_state, *ovf = d_state + nq, *ovf_list = d_state + 2 * (size_t)nq,
           *ovf_count = d_state + 3 * (size_t)nq, *n_f64 = ovf_count + 1, *spill_count = ovf_count + 2;
  // spill list (big-query indices for the large merge): spill_count + 1 .. + nq
  if ((rc = launch_fill_u32(T_global, nq, f32_sortable(INFINITY), st))) return rc;
  FKNN_CUDA(cudaMemsetAsync(ovf, 0, (size_t)nq * 4, st));
  FKNN_CUDA(cudaMemsetAsync(ovf_count, 0, 12, st));
  // pilot state: bound estimate, seeded flag, pilot overflow per query
  uint32_t *d_pilot = nullptr, *seeded = nullptr;
  if (tune.pilot_stride > 1) {
    if ((rc = ws_get(idx, 11, (size_t)nq * 12, (void **)&d_pilot))) return rc;
    seeded = d_pilot + nq;
    FKNN_CUDA(cudaMemsetAsync(seeded, 0, (size_t)nq * 4, st));
  }
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (stats)
    for (auto &e : ev) FKNN_CUDA(cudaEventCreate(&e));
  const OrderData &OT = idx->ord[ORDER_TIME], &OC = idx->ord[ORDER_CAT];
  if (nitems) {
    unsigned char *d_at;
    Candidate *d_out;
    uint32_t *d_ocnt;
    float2 *d_lqs;
    if ((rc = ws_get(idx, 4, (size_t)ntile * TB, (void **)&d_at))) return rc;
    if ((rc = ws_get(idx, 10, (size_t)ntile * BQ * sizeof(float2), (void **)&d_lqs))) return rc;
    if ((rc = ws_get(idx, 6, (size_t)nitems * BQ * capb * sizeof(Candidate), (void **)&d_out))) return rc;
    if ((rc = ws_get(idx, 7, (size_t)nitems * BQ * 4, (void **)&d_ocnt))) return rc;
    LaneSrc ls;
    ls.lane_q = (const int32_t *)(d_blob + o_lq);
    ls.lane_s = (const uint32_t *)(d_blob + o_ls);
    ls.lane_e = (const uint32_t *)(d_blob + o_le);
    if constexpr (F::kFP8)
      k_tile_stage_fp8<<<ntile, 256, 0, st>>>(d_q, ls, (const Tile *)(d_blob + o_tiles), ntile, idx->fp8_scale,
                                              idx->fp8_scale + DIM, d_at, d_lqs);
    else
      k_tile_stage_bf16<<<ntile, 256, 0, st>>>(d_q, ls, (const Tile *)(d_blob + o_tiles), ntile, d_desc,
                                               (__nv_bfloat16 *)d_at, d_lqs);
    // per device context, so set on every call (cheap)
    // the compaction holds a whole list in registers: 32 x NPL >= capb
    auto screen = capb <= 512 ? k_screen_tc<F, 16> : capb <= 768 ? k_screen_tc<F, 24>
                : capb <= 1024 ? k_screen_tc<F, 32> : k_screen_tc<F, 40>;
    FKNN_CUDA(cudaFuncSetAttribute(screen, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sizeof(BScreenSmem<F>)));
    FKNN_CUDA(cudaFuncSetAttribute(k_merge_rerank<RR_CAP_SMALL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sizeof(RerankSmem<RR_CAP_SMALL>)));
    FKNN_CUDA(cudaFuncSetAttribute(k_merge_rerank<RR_CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sizeof(RerankSmem<RR_CAP>)));
    if (stats) FKNN_CUDA(cudaEventRecord(ev[0], st));
    void *const *blocks = F::kFP8 ? idx->fp8_blocks : idx->bf16_blocks;
    const uint32_t stride = tune.pilot_stride;
    if (stride > 1) {
      // pilot: every stride-th row block with a short list; its r-th
      // distance seeds the bound of queries with long slabs
      // the k'-th of all rows ranks about k'/stride in the sample; r = 3 k'/stride
      // + 8 lies above it but for a vanishing fraction of queries
      const uint32_t r = std::min<uint32_t>(kprime, (3 * kprime + stride - 1) / stride + 8);
      uint32_t *T_A = d_pilot, *ovf_A = d_pilot + 2 * (size_t)nq;
      if ((rc = launch_fill_u32(T_A, nq, f32_sortable(INFINITY), st))) return rc;
      FKNN_CUDA(cudaMemsetAsync(ovf_A, 0, (size_t)nq * 4, st));
      screen<<<nitems, B_THREADS, sizeof(BScreenSmem<F>), st>>>(
          (const WorkItem *)(d_blob + o_items), (const Tile *)(d_blob + o_tiles), d_at, ls, d_lqs,
          (const unsigned char *)blocks[ORDER_TIME], (const unsigned char *)blocks[ORDER_CAT], T_A, ovf_A, d_out,
          d_ocnt, r, capb, 0, stride, 0u, nitems, nullptr, nullptr, nullptr, idx->d_flag);
      k_seed_bounds<<<std::max<uint32_t>(1, std::min<uint32_t>((nbig + 255) / 256, 1184)), 256, 0, st>>>(
          (const uint32_t *)(d_blob + o_big), nbig, nullptr, d_desc, T_A, ovf_A, 16 * stride * BR, T_global, seeded);
      g_launches += 3;
    }
    screen<<<nitems, B_THREADS, sizeof(BScreenSmem<F>), st>>>(
        (const WorkItem *)(d_blob + o_items), (const Tile *)(d_blob + o_tiles), d_at, ls, d_lqs,
        (const unsigned char *)blocks[ORDER_TIME], (const unsigned char *)blocks[ORDER_CAT], T_global, ovf, d_out,
        d_ocnt, kprime, capb, tune.bound_refresh, 1, idx->test_withhold ? 1u : 0u, nitems, nullptr, nullptr, nullptr,
        idx->d_flag);
    idx->test_withhold = false;
    if (stats) FKNN_CUDA(cudaEventRecord(ev[1], st));
    MergeArgs A;
    A.big_q = (const uint32_t *)(d_blob + o_big);
    A.big_tile = (const uint32_t *)(d_blob + o_btile);
    A.big_lane = (const uint32_t *)(d_blob + o_blane);
    A.tiles = (const Tile *)(d_blob + o_tiles);
    A.item_slot = (const uint32_t *)(d_blob + o_slot);
    A.out = d_out;
    A.out_cnt = d_ocnt;
    A.desc = d_desc;
    A.q = d_q;
    A.vecs = idx->vecs;
    A.perm_t = OT.perm;
    A.perm_c = OC.perm;
    A.ovf = ovf;
    A.ovf_list = ovf_list;
    A.ovf_count = ovf_count;
    A.k = k;
    A.kprime = kprime;
    A.capb = capb;
    A.seeded = stride > 1 ? seeded : nullptr;
    A.ids = d_ids;
    A.dists = d_dists;
    A.n_f64 = n_f64;
    A.nbig_d = nullptr;
    // queries with more candidates than the common merge holds go to the large one
    uint32_t *spill = spill_count + 1;
    k_merge_rerank<RR_CAP_SMALL><<<nbig, RR_THREADS, sizeof(RerankSmem<RR_CAP_SMALL>), st>>>(
        A, nbig, nullptr, nullptr, spill, spill_count);
    k_merge_rerank<RR_CAP><<<148 * 2, RR_THREADS, sizeof(RerankSmem<RR_CAP>), st>>>(A, 0, spill, spill_count,
                                                                                     nullptr, nullptr);
    g_launches += 4;
  }
  if (stats) FKNN_CUDA(cudaEventRecord(ev[2], st));
  if (nbig)
    if ((rc = launch_exact_scan(idx, ovf_list, ovf_count, 0, 148 * 2, d_desc, d_q, k, d_ids, d_dists, st))) return rc;
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
    uint32_t h2[2] = {0, 0};
    FKNN_CUDA(cudaMemcpyAsync(h2, ovf_count, 8, cudaMemcpyDeviceToHost, st));
    FKNN_CUDA(cudaStreamSynchronize(st));
    stats->n_overflow = h2[0];
    stats->n_boundary_f64 = h2[1];
  }
  return FKNN_OK;
}

// The same search with the plan built on the device (device_plan.cu) and
// every launch of fixed size, captured once into a CUDA graph and replayed
// while nq, k, k', the tuning, the pointers and the scratch buffers stay
// the same.  Screens run persistent over the device item count; merges and
// scans read their counts from device memory.
template <class F>
static int search_tc_graph(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k,
                           uint32_t kprime, uint32_t *d_ids, float *d_dists, cudaStream_t st,
                           fknn_search_stats *stats) {
  constexpr uint32_t TB = Tiles<F>::BYTES;
  int rc;
  const fknn_tuning tune = idx->tuning[F::kFP8 ? FKNN_MODE_FP8_RERANK : FKNN_MODE_BF16_RERANK];
  const uint32_t capb =
      (uint32_t)std::min<size_t>(1280, align_up(kprime + std::max<uint32_t>(tune.list_slack, 2 * BR), 128));
  PlanShape shape;
  shape.tq = BQ;
  shape.blk_rows = BR;
  shape.small_slab = SMALL_SLAB;
  shape.min_chunk_blocks = tune.min_chunk_blocks;
  shape.target_items = idx->num_sms * tune.items_per_sm;
  DevPlanSizes z = device_plan_sizes(idx, nq, shape);
  const uint64_t per_item = (uint64_t)BQ * capb * sizeof(Candidate);
  shape.max_items_per_tile = (uint32_t)std::max<uint64_t>(
      1, std::min<uint64_t>(RR_CAP / capb, (8ull << 30) / (per_item * z.ntile_max)));
  // all buffers exist before the capture (a capture may not allocate)
  QueryDesc *d_desc;
  void *d_plan;
  unsigned char *d_at;
  float2 *d_lqs;
  Candidate *d_out;
  uint32_t *d_ocnt, *d_state, *d_pilot = nullptr;
  if ((rc = ws_get(idx, 2, (size_t)nq * sizeof(QueryDesc), (void **)&d_desc))) return rc;
  if ((rc = ws_get(idx, 19, device_plan_bytes(nq, z), &d_plan))) return rc;
  if ((rc = ws_get(idx, 4, (size_t)z.ntile_max * TB, (void **)&d_at))) return rc;
  if ((rc = ws_get(idx, 10, (size_t)z.ntile_max * BQ * sizeof(float2), (void **)&d_lqs))) return rc;
  if ((rc = ws_get(idx, 6, (size_t)z.nitems_max * per_item, (void **)&d_out))) return rc;
  if ((rc = ws_get(idx, 7, (size_t)z.nitems_max * BQ * 4, (void **)&d_ocnt))) return rc;
  if ((rc = ws_get(idx, 5, (size_t)nq * 16 + 64, (void **)&d_state))) return rc;
  const uint32_t stride = tune.pilot_stride;
  if (stride > 1 && (rc = ws_get(idx, 11, (size_t)nq * 12, (void **)&d_pilot))) return rc;
  {  // the radix sort's histogram slot at its largest (the plan sorts nq keys)
    void *h;
    const size_t keys = std::max<size_t>(nq, z.nitems_max);  // ... and the work items
    if ((rc = ws_get(idx, 15, ((keys + 4095) / 4096) * 256 * sizeof(uint32_t) + 256, &h))) return rc;
  }
  DevPlan P;
  device_plan_layout(P, d_plan, nq, z);
  auto screen = capb <= 512 ? k_screen_tc<F, 16> : capb <= 768 ? k_screen_tc<F, 24>
              : capb <= 1024 ? k_screen_tc<F, 32> : k_screen_tc<F, 40>;
  FKNN_CUDA(cudaFuncSetAttribute(screen, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(BScreenSmem<F>)));
  FKNN_CUDA(cudaFuncSetAttribute(k_merge_rerank<RR_CAP_SMALL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(RerankSmem<RR_CAP_SMALL>)));
  FKNN_CUDA(cudaFuncSetAttribute(k_merge_rerank<RR_CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(RerankSmem<RR_CAP>)));
  GraphCache &G = idx->graph;
  const bool withhold = idx->test_withhold;
  idx->test_withhold = false;
  const std::vector<uint64_t> key = {
      (uint64_t)F::kFP8, nq, k, kprime, capb, tune.list_slack, tune.items_per_sm, tune.min_chunk_blocks,
      tune.bound_refresh, tune.pilot_stride, (uint64_t)withhold, (uint64_t)(uintptr_t)d_q, (uint64_t)(uintptr_t)d_meta,
      (uint64_t)(uintptr_t)d_ids, (uint64_t)(uintptr_t)d_dists, (uint64_t)(uintptr_t)d_desc,
      (uint64_t)(uintptr_t)d_plan, (uint64_t)(uintptr_t)d_at, (uint64_t)(uintptr_t)d_lqs, (uint64_t)(uintptr_t)d_out,
      (uint64_t)(uintptr_t)d_ocnt, (uint64_t)(uintptr_t)d_state, (uint64_t)(uintptr_t)d_pilot,
      (uint64_t)(uintptr_t)idx->ws[15].p};
  if (!G.exec || G.key != key) {
    G.release();
    for (auto &e : G.ev) FKNN_CUDA(cudaEventCreate(&e));
    if (!G.cap) FKNN_CUDA(cudaStreamCreateWithFlags(&G.cap, cudaStreamNonBlocking));
    if (!G.side) FKNN_CUDA(cudaStreamCreateWithFlags(&G.side, cudaStreamNonBlocking));
    if (!G.fork) FKNN_CUDA(cudaEventCreateWithFlags(&G.fork, cudaEventDisableTiming));
    if (!G.join) FKNN_CUDA(cudaEventCreateWithFlags(&G.join, cudaEventDisableTiming));
    const uint32_t l0 = g_launches;
    const cudaStream_t user_st = st;
    st = G.cap;  // captured nodes carry no stream: the replay goes to the caller's
    FKNN_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    // everything below is enqueued only; a failure ends the capture first
    auto body = [&]() -> int {
      int r;
      if ((r = enqueue_query_prep(idx, d_q, d_meta, nq, d_desc, st))) return r;
      if ((r = device_plan_build(idx, d_desc, d_meta, P, shape, st))) return r;
      // the short-slab exact scans need only the plan's list: a branch of
      // the graph beside the contraction (their rows of ids / dists are
      // disjoint from the merge's)
      FKNN_CUDA(cudaEventRecord(G.fork, st));
      FKNN_CUDA(cudaStreamWaitEvent(G.side, G.fork, 0));
      if ((r = launch_exact_scan(idx, P.small, P.cnt + DP_NSMALL, 0, 148 * 8, d_desc, d_q, k, d_ids, d_dists,
                                 G.side)))
        return r;
      FKNN_CUDA(cudaEventRecord(G.join, G.side));
      uint32_t *T_global = d_state, *ovf = d_state + nq, *ovf_list = d_state + 2 * (size_t)nq,
               *ovf_count = d_state + 3 * (size_t)nq, *n_f64 = ovf_count + 1, *spill_count = ovf_count + 2;
      if ((r = launch_fill_u32(T_global, nq, f32_sortable(INFINITY), st))) return r;
      FKNN_CUDA(cudaMemsetAsync(ovf, 0, (size_t)nq * 4, st));
      FKNN_CUDA(cudaMemsetAsync(ovf_count, 0, 12, st));
      const OrderData &OT = idx->ord[ORDER_TIME], &OC = idx->ord[ORDER_CAT];
      LaneSrc ls;
      ls.tile_first = P.tile_first;
      ls.order_q = P.vals;
      ls.desc = d_desc;
      ls.ntile = P.cnt + DP_NTILE;
      const unsigned tgrid = std::min<uint32_t>(z.ntile_max, (uint32_t)idx->num_sms * 4);
      if constexpr (F::kFP8)
        k_tile_stage_fp8<<<tgrid, 256, 0, st>>>(d_q, ls, P.tiles, 0, idx->fp8_scale, idx->fp8_scale + DIM, d_at,
                                                d_lqs);
      else
        k_tile_stage_bf16<<<tgrid, 256, 0, st>>>(d_q, ls, P.tiles, 0, d_desc, (__nv_bfloat16 *)d_at, d_lqs);
      g_launches += 1;
      FKNN_CUDA(cudaEventRecordWithFlags(G.ev[0], st, cudaEventRecordExternal));  // an event node of the graph
      void *const *blocks = F::kFP8 ? idx->fp8_blocks : idx->bf16_blocks;
      const unsigned sgrid = std::min<uint32_t>(z.nitems_max, (uint32_t)idx->num_sms * 2);
      uint32_t *seeded = nullptr;
      if (stride > 1) {
        const uint32_t rr = std::min<uint32_t>(kprime, (3 * kprime + stride - 1) / stride + 8);
        uint32_t *T_A = d_pilot, *ovf_A = d_pilot + 2 * (size_t)nq;
        seeded = d_pilot + nq;
        FKNN_CUDA(cudaMemsetAsync(seeded, 0, (size_t)nq * 4, st));
        if ((r = launch_fill_u32(T_A, nq, f32_sortable(INFINITY), st))) return r;
        FKNN_CUDA(cudaMemsetAsync(ovf_A, 0, (size_t)nq * 4, st));
        screen<<<sgrid, B_THREADS, sizeof(BScreenSmem<F>), st>>>(
            P.items, P.tiles, d_at, ls, d_lqs, (const unsigned char *)blocks[ORDER_TIME],
            (const unsigned char *)blocks[ORDER_CAT], T_A, ovf_A, d_out, d_ocnt, rr, capb, 0, stride, 0u, 0,
            P.cnt + DP_NITEMS, P.ord_val, P.queue, idx->d_flag);
        k_seed_bounds<<<1184, 256, 0, st>>>(P.big_q, 0, P.cnt + DP_NBIG, d_desc, T_A, ovf_A, 16 * stride * BR,
                                            T_global, seeded);
        g_launches += 2;
      }
      screen<<<sgrid, B_THREADS, sizeof(BScreenSmem<F>), st>>>(
          P.items, P.tiles, d_at, ls, d_lqs, (const unsigned char *)blocks[ORDER_TIME],
          (const unsigned char *)blocks[ORDER_CAT], T_global, ovf, d_out, d_ocnt, kprime, capb, tune.bound_refresh, 1,
          withhold ? 1u : 0u, 0, P.cnt + DP_NITEMS, P.ord_val, P.queue + 1, idx->d_flag);
      g_launches += 1;
      FKNN_CUDA(cudaEventRecordWithFlags(G.ev[1], st, cudaEventRecordExternal));  // an event node of the graph
      MergeArgs A;
      A.big_q = P.big_q;
      A.big_tile = P.big_tile;
      A.big_lane = P.big_lane;
      A.tiles = P.tiles;
      A.item_slot = nullptr;  // a tile's items are consecutive
      A.out = d_out;
      A.out_cnt = d_ocnt;
      A.desc = d_desc;
      A.q = d_q;
      A.vecs = idx->vecs;
      A.perm_t = OT.perm;
      A.perm_c = OC.perm;
      A.ovf = ovf;
      A.ovf_list = ovf_list;
      A.ovf_count = ovf_count;
      A.k = k;
      A.kprime = kprime;
      A.capb = capb;
      A.seeded = seeded;
      A.ids = d_ids;
      A.dists = d_dists;
      A.n_f64 = n_f64;
      A.nbig_d = P.cnt + DP_NBIG;
      uint32_t *spill = spill_count + 1;
      k_merge_rerank<RR_CAP_SMALL><<<std::min<uint32_t>(nq, (uint32_t)idx->num_sms * 32), RR_THREADS,
                                     sizeof(RerankSmem<RR_CAP_SMALL>), st>>>(A, 0, nullptr, nullptr, spill,
                                                                             spill_count);
      k_merge_rerank<RR_CAP><<<148 * 2, RR_THREADS, sizeof(RerankSmem<RR_CAP>), st>>>(A, 0, spill, spill_count,
                                                                                       nullptr, nullptr);
      g_launches += 2;
      FKNN_CUDA(cudaEventRecordWithFlags(G.ev[2], st, cudaEventRecordExternal));  // an event node of the graph
      if ((r = launch_exact_scan(idx, ovf_list, ovf_count, 0, 148 * 2, d_desc, d_q, k, d_ids, d_dists, st))) return r;
      FKNN_CUDA(cudaStreamWaitEvent(st, G.join, 0));
      FKNN_CUDA(cudaEventRecordWithFlags(G.ev[3], st, cudaEventRecordExternal));  // an event node of the graph
      FKNN_CUDA(cudaGetLastError());
      return FKNN_OK;
    };
    const int brc = body();
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    st = user_st;
    if (brc || ce != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      G.release();
      cudaGetLastError();
      return brc ? brc : cuda_fail(ce, "cudaStreamEndCapture");
    }
    const cudaError_t ie = cudaGraphInstantiate(&G.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      G.exec = nullptr;
      G.release();
      return cuda_fail(ie, "cudaGraphInstantiate");
    }
    G.key = key;
    G.launches = g_launches - l0;
    st = user_st;
  }
  g_launches = G.launches;
  FKNN_CUDA(cudaGraphLaunch(G.exec, st));
  int flag = 0;
  FKNN_CUDA(cudaMemcpyAsync(&flag, idx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  if ((rc = check_query_flag_value(flag & ~ERR_WAIT_TIMEOUT))) return rc;
  if (stats) {
    float ms = 0.f;
    FKNN_CUDA(cudaEventElapsedTime(&ms, G.ev[0], G.ev[1]));
    stats->ms_screen = ms;
    FKNN_CUDA(cudaEventElapsedTime(&ms, G.ev[1], G.ev[2]));
    stats->ms_merge = ms;
    FKNN_CUDA(cudaEventElapsedTime(&ms, G.ev[2], G.ev[3]));
    stats->ms_scan = ms;
    uint32_t c[16];
    FKNN_CUDA(cudaMemcpy(c, P.cnt, sizeof(c), cudaMemcpyDeviceToHost));
    uint32_t h2[2] = {0, 0};
    FKNN_CUDA(cudaMemcpy(h2, d_state + 3 * (size_t)nq, 8, cudaMemcpyDeviceToHost));
    auto u64 = [&](int i) { return (uint64_t)c[i] | ((uint64_t)c[i + 1] << 32); };
    stats->pairs_screened = u64(10);
    stats->pairs_passing = u64(12);
    stats->pairs_contraction = u64(14);
    stats->n_tiles = c[DP_NTILE];
    stats->n_work_items = c[DP_NITEMS];
    stats->n_small = c[DP_NSMALL];
    stats->ms_plan = 0.f;
    stats->n_overflow = h2[0];
    stats->n_boundary_f64 = h2[1];
  }
  return FKNN_OK;
}

int search_bf16(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k, uint32_t kprime,
                uint32_t *d_ids, float *d_dists, cudaStream_t st, fknn_search_stats *stats) {
  return search_tc<FmtBF16>(idx, d_q, d_meta, nq, k, kprime, d_ids, d_dists, st, stats);
}

int search_bf16_graph(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k,
                      uint32_t kprime, uint32_t *d_ids, float *d_dists, cudaStream_t st, fknn_search_stats *stats) {
  return search_tc_graph<FmtBF16>(idx, d_q, d_meta, nq, k, kprime, d_ids, d_dists, st, stats);
}

int search_fp8_graph(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k,
                     uint32_t kprime, uint32_t *d_ids, float *d_dists, cudaStream_t st, fknn_search_stats *stats) {
  return search_tc_graph<FmtFP8>(idx, d_q, d_meta, nq, k, kprime, d_ids, d_dists, st, stats);
}

int search_fp8(fknn_index *idx, const float *d_q, const float *d_meta, uint32_t nq, uint32_t k, uint32_t kprime,
               uint32_t *d_ids, float *d_dists, cudaStream_t st, fknn_search_stats *stats) {
  return search_tc<FmtFP8>(idx, d_q, d_meta, nq, k, kprime, d_ids, d_dists, st, stats);
}

}  // namespace fknn
