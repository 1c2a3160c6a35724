// Predicate evaluation + row compaction over the attribute columns: the
// per-row predicate of utils.h:98-137 (type 0 every row, 1 int32(label) ==
// int32(v), 2 l <= ts <= r, 3 both) applied to whole columns, writing each
// predicate's passing row ids in increasing order.
//
// One pass over the columns for up to FP_MAXP predicates (k_filter_scan,
// a single-pass scan):
//   * a CTA takes the next 4,096-row tile from a ticket counter, so every
//     tile before it is already running or done;
//   * its threads load the tile's labels and timestamps as float4 (16 rows
//     each, coalesced) and evaluate every predicate on them;
//   * per predicate the tile publishes its passing count at once, then sums
//     the counts of all the tiles before it (each thread a strided share, so
//     no tile waits on another tile's prefix: only on counts published
//     right after their loads), and every passing row writes its id at
//     prefix + its rank in the tile.
// A status word holds its flag and its value together, so one 64-bit
// volatile load sees a consistent pair.  The waits are bounded by the
// global timer; a tile that gives up makes that predicate's count
// UINT64_MAX.  Nothing is read back: the counts land in device memory, so
// a batch of calls streams back to back.  Algorithmic traffic per launch:
// 8 B per row plus 4 B per passing row.
#include <algorithm>
#include <cstring>

#include "device_util.cuh"

namespace fknn {

namespace {

constexpr int FS_THREADS = 256;
constexpr int FS_NW = FS_THREADS / 32;
constexpr int FS_IT = 4;                          // float4 loads per column per thread
constexpr int FS_TILE = FS_THREADS * 4 * FS_IT;   // 4,096 rows per tile
constexpr int FS_SEG = FS_IT * FS_NW;             // 128-row warp segments per tile (= 32)
constexpr uint32_t FP_MAXP = 16;                  // predicates per launch
constexpr uint64_t ST_AGG = 1ull << 62, ST_FLAGS = 3ull << 62;
constexpr uint32_t FS_UNROLL = 4;                 // status words in flight per thread

static_assert(FS_SEG == 32, "one warp scans the tile's segments");

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

__device__ __forceinline__ uint64_t ld_volatile_u64(const uint64_t *p) { return *(const volatile uint64_t *)p; }

// status: np x ntiles words and the ticket after them, zeroed before the
// launch.  Grid: ntiles CTAs.
__global__ void __launch_bounds__(FS_THREADS) k_filter_scan(const float *__restrict__ labels,
                                                            const float *__restrict__ ts, uint64_t n,
                                                            FilterPreds P, uint32_t np, uint32_t ntiles,
                                                            uint64_t *__restrict__ status, uint32_t *ticket,
                                                            uint32_t *__restrict__ out, uint64_t out_stride,
                                                            uint64_t *__restrict__ counts) {
  __shared__ float4 pm[FP_MAXP];
  __shared__ uint32_t seg[FS_SEG];
  __shared__ uint32_t s_tile, s_total;
  __shared__ uint64_t s_prefix, s_part[FS_NW];
  __shared__ int s_fail[FS_NW];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid < (int)FP_MAXP) pm[tid] = P.m[tid];
  if (tid == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const uint32_t t = s_tile;
  const uint64_t base = (uint64_t)t * FS_TILE;
  // this thread's rows: base + it*1024 + 4*tid + c, c = 0..3
  int32_t lab[FS_IT][4];
  float tv[FS_IT][4];
  uint32_t valid = 0;  // bit it*4+c: the row is inside the base
#pragma unroll
  for (int it = 0; it < FS_IT; ++it) {
    const uint64_t r = base + (uint64_t)it * (FS_THREADS * 4) + 4 * tid;
    if (r + 4 <= n) {
      const float4 a = __ldcs(reinterpret_cast<const float4 *>(labels + r));
      const float4 b = __ldcs(reinterpret_cast<const float4 *>(ts + r));
      lab[it][0] = (int32_t)a.x;
      lab[it][1] = (int32_t)a.y;
      lab[it][2] = (int32_t)a.z;
      lab[it][3] = (int32_t)a.w;
      tv[it][0] = b.x;
      tv[it][1] = b.y;
      tv[it][2] = b.z;
      tv[it][3] = b.w;
      valid |= 0xfu << (it * 4);
    } else {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        lab[it][c] = 0;
        tv[it][c] = 0.f;
        if (r + c < n) {
          lab[it][c] = (int32_t)labels[r + c];
          tv[it][c] = ts[r + c];
          valid |= 1u << (it * 4 + c);
        }
      }
    }
  }
  for (uint32_t p = 0; p < np; ++p) {
    const float4 m = pm[p];
    uint32_t mask = 0;
#pragma unroll
    for (int it = 0; it < FS_IT; ++it)
#pragma unroll
      for (int c = 0; c < 4; ++c) mask |= (pred_pass(m, lab[it][c], tv[it][c]) ? 1u : 0u) << (it * 4 + c);
    mask &= valid;
    // rank of this lane's rows inside its warp's 128-row segment of each it
    uint32_t excl[FS_IT];
#pragma unroll
    for (int it = 0; it < FS_IT; ++it) {
      const uint32_t cnt = __popc((mask >> (it * 4)) & 0xfu);
      uint32_t inc = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
      }
      excl[it] = inc - cnt;
      if (lane == 31) seg[it * FS_NW + w] = inc;
    }
    __syncthreads();
    uint64_t *st = status + (uint64_t)p * ntiles;
    if (w == 0) {
      // the 32 segments in row order (it-major, then warp): exclusive offsets
      const uint32_t v = seg[lane];
      uint32_t inc = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += x;
      }
      seg[lane] = inc - v;
      if (lane == 31) {
        s_total = inc;
        *(volatile uint64_t *)(st + t) = ST_AGG | inc;  // published before this tile waits on anything
      }
    }
    // the tile's prefix: every thread sums a strided share of the counts the
    // tiles before it published (they took their tickets first, so they run
    // and publish without waiting); the waits are bounded
    uint64_t part = 0;
    bool failed = false;
    const uint64_t t0 = global_ns();
    for (uint32_t j0 = tid; j0 < t && !failed; j0 += FS_UNROLL * FS_THREADS) {
      uint64_t sv[FS_UNROLL];
#pragma unroll
      for (uint32_t u = 0; u < FS_UNROLL; ++u) {
        const uint32_t j = j0 + u * FS_THREADS;
        sv[u] = j < t ? ld_volatile_u64(st + j) : ST_AGG;  // independent loads, in flight together
      }
#pragma unroll
      for (uint32_t u = 0; u < FS_UNROLL; ++u) {
        while (!failed && (sv[u] & ST_FLAGS) == 0) {
          if (global_ns() - t0 > WAIT_NS) failed = true;
          else sv[u] = ld_volatile_u64(st + j0 + u * FS_THREADS);
        }
        part += sv[u] & 0xffffffffull;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    const uint32_t anyfail = __ballot_sync(0xffffffffu, failed);
    if (lane == 0) {
      s_part[w] = part;
      s_fail[w] = anyfail ? 1 : 0;
    }
    __syncthreads();
    if (tid == 0) {
      uint64_t pre = 0;
      int f = 0;
#pragma unroll
      for (int j = 0; j < FS_NW; ++j) {
        pre += s_part[j];
        f |= s_fail[j];
      }
      s_prefix = f ? ~0ull : pre;
      // the count: the last tile's prefix plus its own; a tile that gave up
      // raises it to UINT64_MAX (counts start at 0, combined by max)
      unsigned long long *cp = reinterpret_cast<unsigned long long *>(counts + p);
      if (f) atomicMax(cp, ~0ull);
      else if (t == ntiles - 1) atomicMax(cp, (unsigned long long)(pre + s_total));
    }
    __syncthreads();
    const uint64_t prefix = s_prefix;
    if (prefix != ~0ull) {
      uint32_t *op = out + (uint64_t)p * out_stride;
#pragma unroll
      for (int it = 0; it < FS_IT; ++it) {
        const uint32_t mk = (mask >> (it * 4)) & 0xfu;
        uint32_t pos = (uint32_t)prefix + seg[it * FS_NW + w] + excl[it];
        const uint64_t r = base + (uint64_t)it * (FS_THREADS * 4) + 4 * tid;
#pragma unroll
        for (int c = 0; c < 4; ++c)
          if ((mk >> c) & 1u) op[pos++] = (uint32_t)(r + c);
      }
    }
    __syncthreads();  // seg and s_prefix are rewritten for the next predicate
  }
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
  const uint32_t ntiles = (uint32_t)((n + FS_TILE - 1) / FS_TILE);
  const uint32_t pmax = std::min<uint32_t>(np, FP_MAXP);
  // per launch: status words (predicates x tiles) and the ticket, cleared first
  uint64_t *status;
  int rc;
  if ((rc = ws_get(idx, 16, ((size_t)pmax * ntiles + 1) * sizeof(uint64_t), (void **)&status))) return rc;
  for (uint32_t p0 = 0; p0 < np; p0 += FP_MAXP) {
    const uint32_t m = std::min<uint32_t>(FP_MAXP, np - p0);
    FilterPreds P;
    std::memset(&P, 0, sizeof(P));
    for (uint32_t p = 0; p < m; ++p) {
      const float *q = metas + (size_t)(p0 + p) * 4;
      P.m[p] = make_float4(q[0], q[1], q[2], q[3]);
    }
    uint32_t *ticket = reinterpret_cast<uint32_t *>(status + (size_t)m * ntiles);
    FKNN_CUDA(cudaMemsetAsync(status, 0, ((size_t)m * ntiles + 1) * sizeof(uint64_t), st));
    FKNN_CUDA(cudaMemsetAsync(d_counts + p0, 0, (size_t)m * sizeof(uint64_t), st));
    k_filter_scan<<<ntiles, FS_THREADS, 0, st>>>(idx->labels_f, idx->ts_f, n, P, m, ntiles, status, ticket,
                                                 d_out + (uint64_t)p0 * n, n, d_counts + p0);
    g_launches += 1;
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
  if (tot == ~0ull) {
    set_error("fknn_filter_rows: a bounded device wait gave up");
    return FKNN_ETIMEOUT;
  }
  *count = tot;
  return FKNN_OK;
}

}  // namespace fknn
