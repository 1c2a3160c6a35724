// Predicate evaluation + row compaction over the attribute columns: the
// per-row predicate of utils.h:98-137 (type 0 every row, 1 int32(label) ==
// int32(v), 2 l <= ts <= r, 3 both) applied to whole columns, writing each
// predicate's passing row ids in increasing order.
//
// Two launches, and the columns are read once for up to FP_MAXP predicates:
//   k_filter_mark  each CTA owns one contiguous, equal row range; per
//                  2,048-row chunk every thread loads 8 labels and 8
//                  timestamps (coalesced), and every predicate's warp ballots
//                  are stored as a bit per row (N/8 bytes per predicate,
//                  which stays in L2) plus the CTA's passing count;
//   k_filter_emit  per (CTA range, predicate): the sum of the counts of the
//                  ranges before it, then per chunk a scan of the 64 words'
//                  popcounts, and every passing row writes its id at
//                  base + word offset + its rank inside the word.
// Nothing is read back: the counts land in device memory, so a batch of
// calls streams back to back.  Algorithmic traffic per launch: 8 B per row
// plus 4 B per passing row; the kernels add N/4 bytes per predicate of
// bit-array traffic, mostly in L2.
#include <algorithm>
#include <cstring>

#include "device_util.cuh"

namespace fknn {

namespace {

constexpr int FP_THREADS = 256;
constexpr int FP_ITEMS = 8;
constexpr int FP_CHUNK = FP_THREADS * FP_ITEMS;  // rows per chunk
constexpr int FP_WORDS = FP_CHUNK / 32;          // bit words per chunk
constexpr int FP_NW = FP_THREADS / 32;
constexpr uint32_t FP_MAXP = 16;                 // predicates per launch
constexpr int FP_CTAS_PER_SM = 8;                // resident at <= 32 registers: one wave

struct FilterPreds {
  float4 m[FP_MAXP];  // (type, v, l, r), checked on the host
};

__device__ __forceinline__ bool pred_pass(const float4 &m, int32_t lab, float t) {
  const uint32_t type = (uint32_t)m.x;
  const int32_t v = (int32_t)m.y;
  switch (type) {
    case 0: return true;
    case 1: return lab == v;
    case 2: return t >= m.z && t <= m.w;
    default: return lab == v && t >= m.z && t <= m.w;
  }
}

__global__ void __launch_bounds__(FP_THREADS, FP_CTAS_PER_SM) k_filter_mark(const float *__restrict__ labels,
                                                            const float *__restrict__ ts, uint64_t n,
                                                            FilterPreds P, uint32_t np, uint64_t rows_per_cta,
                                                            uint32_t *__restrict__ bits, uint64_t words_per_pred,
                                                            uint32_t *__restrict__ cta_cnt) {
  __shared__ uint32_t wcnt[FP_MAXP][FP_NW];
  __shared__ float4 pm[FP_MAXP];  // the predicates, indexed at run time (kept out of local memory)
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int i = tid; i < (int)(FP_MAXP * FP_NW); i += FP_THREADS) (&wcnt[0][0])[i] = 0;
  if (tid < (int)FP_MAXP) pm[tid] = P.m[tid];
  __syncthreads();
  const uint64_t r0 = (uint64_t)blockIdx.x * rows_per_cta;
  const uint64_t r1 = min(n, r0 + rows_per_cta);
  for (uint64_t c0 = r0; c0 < r1; c0 += FP_CHUNK) {
    int32_t lab[FP_ITEMS];
    float t[FP_ITEMS];
#pragma unroll
    for (int i = 0; i < FP_ITEMS; ++i) {
      const uint64_t r = c0 + (uint64_t)i * FP_THREADS + tid;
      lab[i] = 0;
      t[i] = 0.f;
      if (r < r1) {
        lab[i] = (int32_t)__ldcs(labels + r);
        t[i] = __ldcs(ts + r);
      }
    }
    for (uint32_t p = 0; p < np; ++p) {
      const float4 m = pm[p];
      uint32_t mine = 0, cnt = 0;
#pragma unroll
      for (int i = 0; i < FP_ITEMS; ++i) {
        const uint64_t r = c0 + (uint64_t)i * FP_THREADS + tid;
        const uint32_t b = __ballot_sync(0xffffffffu, r < r1 && pred_pass(m, lab[i], t[i]));
        if (lane == i) mine = b;
        cnt += __popc(b);
      }
      // word of rows c0 + lane*256 + w*32 .. +31
      if (lane < FP_ITEMS && c0 + (uint64_t)lane * FP_THREADS + w * 32 < r1)
        bits[p * words_per_pred + c0 / 32 + lane * FP_NW + w] = mine;
      if (lane == 0) wcnt[p][w] += cnt;
    }
  }
  __syncthreads();
  if (tid < (int)np) {
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < FP_NW; ++j) s += wcnt[tid][j];
    cta_cnt[(uint64_t)tid * gridDim.x + blockIdx.x] = s;
  }
}

// Block-wide sum of one value per thread (all threads get it).
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t *red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) red[w] = v;
  __syncthreads();
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < FP_NW; ++j) s += red[j];
  __syncthreads();
  return s;
}

__global__ void __launch_bounds__(FP_THREADS) k_filter_emit(uint64_t n, uint64_t rows_per_cta,
                                                            const uint32_t *__restrict__ bits, uint64_t words_per_pred,
                                                            const uint32_t *__restrict__ cta_cnt,
                                                            uint32_t *__restrict__ out, uint64_t out_stride,
                                                            uint64_t *__restrict__ counts) {
  __shared__ uint32_t red[FP_NW];
  __shared__ uint32_t wsm[FP_WORDS], woff[FP_WORDS + 1];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t g = blockIdx.x, G = gridDim.x, p = blockIdx.y;
  const uint32_t *cc = cta_cnt + (uint64_t)p * G;
  uint32_t s = 0;
  for (uint32_t j = tid; j < g; j += FP_THREADS) s += cc[j];
  uint32_t base = block_sum(s, red);
  const uint64_t r0 = (uint64_t)g * rows_per_cta;
  const uint64_t r1 = min(n, r0 + rows_per_cta);
  const uint32_t *bp = bits + (uint64_t)p * words_per_pred;
  uint32_t *op = out + (uint64_t)p * out_stride;
  const uint32_t lt = (1u << lane) - 1u;
  for (uint64_t c0 = r0; c0 < r1; c0 += FP_CHUNK) {
    // exclusive scan of the chunk's FP_WORDS word popcounts
    if (tid < FP_WORDS) {
      const uint32_t word = (c0 + (uint64_t)tid * 32 < r1) ? __ldcs(bp + c0 / 32 + tid) : 0u;
      const uint32_t pc = __popc(word);
      uint32_t inc = pc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
      }
      wsm[tid] = word;
      woff[tid] = inc - pc;
      if (lane == 31) red[w] = inc;
    }
    __syncthreads();
    if (tid < FP_WORDS) {
      uint32_t add = 0;
      for (int j = 0; j < w; ++j) add += red[j];
      woff[tid] += add;
      if (tid == FP_WORDS - 1) woff[FP_WORDS] = woff[tid] + __popc(wsm[tid]);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < FP_ITEMS; ++i) {
      const int wi = i * FP_NW + w;
      const uint32_t word = wsm[wi];
      if ((word >> lane) & 1u)
        op[base + woff[wi] + __popc(word & lt)] = (uint32_t)(c0 + (uint64_t)i * FP_THREADS + tid);
    }
    base += woff[FP_WORDS];
    __syncthreads();
  }
  if (g == G - 1 && tid == 0) counts[p] = base;
}

}  // namespace

int filter_check_preds(const float *metas, uint32_t np, const char *who) {
  for (uint32_t p = 0; p < np; ++p) {
    const float *m = metas + (size_t)p * 4;
    const float t = m[0];
    if (!(t == 0.f || t == 1.f || t == 2.f || t == 3.f)) {
      set_error(std::string(who) + ": query type not in {0,1,2,3}");
      return FKNN_EINVAL;
    }
    if ((t == 1.f || t == 3.f) && !(fabsf(m[1]) < 2147483648.f)) {
      set_error(std::string(who) + ": category outside int32");
      return FKNN_EINVAL;
    }
  }
  return FKNN_OK;
}

// np predicates (host memory, checked) over the index's original-order
// columns; out_ids row p (stride n) and counts[p] are device memory.
int filter_rows_batch(fknn_index *idx, const float *metas, uint32_t np, uint32_t *d_out, uint64_t *d_counts,
                      cudaStream_t st) {
  const uint64_t n = idx->n;
  if (np == 0) return FKNN_OK;
  // equal row ranges, a multiple of 256 rows each, one resident wave of CTAs
  const uint64_t g0 = std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)idx->num_sms * FP_CTAS_PER_SM,
                                                                (n + FP_THREADS - 1) / FP_THREADS));
  const uint64_t rows_per_cta = ((n + g0 - 1) / g0 + FP_THREADS - 1) / FP_THREADS * FP_THREADS;
  const uint32_t G = (uint32_t)((n + rows_per_cta - 1) / rows_per_cta);
  const uint64_t wpp = (G * rows_per_cta + 31) / 32;
  const uint32_t pmax = std::min<uint32_t>(np, FP_MAXP);
  uint32_t *bits, *cnt;
  int rc;
  if ((rc = ws_get(idx, 16, (size_t)pmax * wpp * 4 + 256, (void **)&bits))) return rc;
  if ((rc = ws_get(idx, 17, (size_t)pmax * G * 4 + 256, (void **)&cnt))) return rc;
  for (uint32_t p0 = 0; p0 < np; p0 += FP_MAXP) {
    const uint32_t m = std::min<uint32_t>(FP_MAXP, np - p0);
    FilterPreds P;
    std::memset(&P, 0, sizeof(P));
    for (uint32_t p = 0; p < m; ++p) {
      const float *q = metas + (size_t)(p0 + p) * 4;
      P.m[p] = make_float4(q[0], q[1], q[2], q[3]);
    }
    k_filter_mark<<<G, FP_THREADS, 0, st>>>(idx->labels_f, idx->ts_f, n, P, m, rows_per_cta, bits, wpp, cnt);
    k_filter_emit<<<dim3(G, m), FP_THREADS, 0, st>>>(n, rows_per_cta, bits, wpp, cnt, d_out + (uint64_t)p0 * n, n,
                                                     d_counts + p0);
    g_launches += 2;
  }
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

// One predicate, its count read back (fknn_filter_rows).
int filter_rows(fknn_index *idx, const float *m4, uint32_t *d_out, uint64_t *count, cudaStream_t st) {
  uint64_t *d_cnt;
  int rc;
  if ((rc = ws_get(idx, 18, 64, (void **)&d_cnt))) return rc;
  if ((rc = filter_rows_batch(idx, m4, 1, d_out, d_cnt, st))) return rc;
  uint64_t tot = 0;
  FKNN_CUDA(cudaMemcpyAsync(&tot, d_cnt, 8, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  *count = tot;
  return FKNN_OK;
}

}  // namespace fknn
