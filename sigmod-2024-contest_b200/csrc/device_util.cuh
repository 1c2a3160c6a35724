// Small device helpers: mbarrier + bulk-copy PTX, bounded waits, sorts,
// the reference's sequential L2.
#pragma once

#include "fknn_internal.cuh"

namespace fknn {

// Every spin-wait gives up after WAIT_NS nanoseconds of the global timer
// (checked every 64 polls), with an iteration cap behind it in case the
// timer does not advance.
constexpr uint64_t WAIT_NS = 1000000000ull;
constexpr uint32_t WAIT_LIMIT = 1u << 28;

// Error bits written to the per-call device flag.
constexpr int ERR_WAIT_TIMEOUT = 1 << 8;
constexpr int ERR_BAD_QUERY_TYPE = 1 << 0;
constexpr int ERR_BAD_QUERY_VALUE = 1 << 1;
constexpr int ERR_BAD_QUERY_VEC = 1 << 2;
constexpr int ERR_PLAN_BOUND = 1 << 3;  // a device-built plan met a buffer bound (reported, never written past)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// 1-D bulk copy global -> shared (the TMA bulk engine), completion counted
// on an mbarrier.  dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait: returns false (and raises ERR_WAIT_TIMEOUT) if the phase
// has not completed within WAIT_NS.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *err) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < WAIT_LIMIT; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63u) == 63u && global_ns() - t0 > WAIT_NS) break;
  }
  atomicOr(err, ERR_WAIT_TIMEOUT);
  return false;
}

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t *p) { return *(const volatile uint32_t *)p; }

// distance.h:62-72 normal_l2(base, query): v = x - q; v *= v; r += v, every
// operation rounded to float, in dimension order, never fused.
__device__ __forceinline__ float seq_l2_strided(const float *x, int xstride, const float *q) {
  float r = 0.f;
#pragma unroll 10
  for (int d = 0; d < DIM; ++d) {
    float v = __fsub_rn(x[d * xstride], q[d]);
    v = __fmul_rn(v, v);
    r = __fadd_rn(r, v);
  }
  return r;
}

__device__ __forceinline__ uint64_t exact_key(float d, uint32_t id) {
  return ((uint64_t)f32_sortable(d) << 32) | id;
}

// In-shared-memory bitonic sort of n (power of two) elements, ascending,
// all threads of the block participate.
template <typename K>
__device__ void block_bitonic_sort(K *key, int n) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < (n >> 1); i += blockDim.x) {
        int lo = 2 * stride * (i / stride) + (i % stride);
        int hi = lo + stride;
        bool asc = (lo & size) == 0;
        K a = key[lo], b = key[hi];
        if ((a > b) == asc) {
          key[lo] = b;
          key[hi] = a;
        }
      }
      __syncthreads();
    }
  }
}

// Key/value variant ordered by (key, val).
template <typename K, typename V>
__device__ void block_bitonic_sort_kv(K *key, V *val, int n) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < (n >> 1); i += blockDim.x) {
        int lo = 2 * stride * (i / stride) + (i % stride);
        int hi = lo + stride;
        bool asc = (lo & size) == 0;
        K a = key[lo], b = key[hi];
        V va = val[lo], vb = val[hi];
        bool gt = (a > b) || (a == b && va > vb);
        if (gt == asc) {
          key[lo] = b;
          key[hi] = a;
          val[lo] = vb;
          val[hi] = va;
        }
      }
      __syncthreads();
    }
  }
}

// Warp-wide bitonic sort of 32*N (key, val) pairs held N per lane, element
// e = j*32 + lane in register j, ascending by (key, val).
template <int N>
__device__ __forceinline__ void warp_bitonic_sort(float (&key)[N], uint32_t (&val)[N]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int size = 2; size <= 32 * N; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
        const int rs = stride >> 5;
#pragma unroll
        for (int j = 0; j < N; ++j) {
          const int p = j ^ rs;
          if (p > j) {
            const bool asc = (((j << 5) | lane) & size) == 0;
            const bool gt = key[j] > key[p] || (key[j] == key[p] && val[j] > val[p]);
            if (gt == asc) {
              float tk = key[j]; key[j] = key[p]; key[p] = tk;
              uint32_t tv = val[j]; val[j] = val[p]; val[p] = tv;
            }
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < N; ++j) {
          const float ok = __shfl_xor_sync(0xffffffffu, key[j], stride);
          const uint32_t ov = __shfl_xor_sync(0xffffffffu, val[j], stride);
          const bool asc = (((j << 5) | lane) & size) == 0;
          const bool lower = (lane & stride) == 0;
          const bool other_less = ok < key[j] || (ok == key[j] && ov < val[j]);
          const bool take_other = (lower == asc) ? other_less : !other_less && !(ok == key[j] && ov == val[j]);
          if (take_other) {
            key[j] = ok;
            val[j] = ov;
          }
        }
      }
    }
  }
}

// L2SqrSQ8_sym (pyglass/glass/simd/distance.hpp:329-366) as an exact int32
// over 112-byte codes: |q - c|^2 = |q|^2 + |c|^2 - 2 q.c with dp4a; qw is the
// query code as 28 words, qq its squared norm.
__device__ __forceinline__ int sq8_dist(const int *__restrict__ qw, int qq, const int8_t *__restrict__ code) {
  const int4 *c4 = reinterpret_cast<const int4 *>(code);
  int cc = 0, qc = 0;
#pragma unroll
  for (int w = 0; w < 28 / 4; ++w) {
    const int4 v = c4[w];
    cc = __dp4a(v.x, v.x, cc);
    cc = __dp4a(v.y, v.y, cc);
    cc = __dp4a(v.z, v.z, cc);
    cc = __dp4a(v.w, v.w, cc);
    qc = __dp4a(qw[4 * w + 0], v.x, qc);
    qc = __dp4a(qw[4 * w + 1], v.y, qc);
    qc = __dp4a(qw[4 * w + 2], v.z, qc);
    qc = __dp4a(qw[4 * w + 3], v.w, qc);
  }
  return qq + cc - 2 * qc;
}


// Offsets of one query's candidate lists in the merge: warp 0 reads the
// item counts (item_slot[item0 + i] selects the item, lane L of tq the
// list) 32 at a time and scans them with shuffles.  prefix[i] = first
// position of item i, *total = their sum, or over_value when there are more
// than max_items items (item_slot NULL: the items are item0 .. item0 +
// nitems - 1).  Caller: the whole block, then __syncthreads().
__device__ __forceinline__ void list_offsets(const uint32_t *__restrict__ item_slot, uint32_t item0, uint32_t nitems,
                                             const uint32_t *__restrict__ out_cnt, uint32_t L, uint32_t tq,
                                             uint32_t *prefix, int *total, uint32_t max_items, int over_value) {
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  if (nitems > max_items) {
    if (lane == 0) *total = over_value;
    return;
  }
  uint32_t carry = 0;
  for (uint32_t base = 0; base < nitems; base += 32) {
    const uint32_t i = base + lane;
    const uint32_t c = i < nitems ? out_cnt[(uint64_t)(item_slot ? item_slot[item0 + i] : item0 + i) * tq + L] : 0u;
    uint32_t inc = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += v;
    }
    if (i < nitems) prefix[i] = carry + inc - c;
    carry += __shfl_sync(0xffffffffu, inc, 31);
  }
  if (lane == 0) *total = (int)carry;
}

}  // namespace fknn
