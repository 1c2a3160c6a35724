// Predicate evaluation + row compaction over the attribute columns: the
// per-row predicate of utils.h:98-137 (type 0 every row, 1 int32(label) ==
// int32(v), 2 l <= ts <= r, 3 both) applied to whole columns, writing each
// predicate's passing row ids in increasing order.
//
// One cooperative launch per group of up to FP_MAXP predicates reads the
// columns once (k_filter_coop).  Every CTA owns a contiguous run of rows
// per round:
//   1. it streams its labels and timestamps (float4 loads, a few steps in
//      flight per warp), evaluates every predicate and keeps, per 128-row
//      warp segment and predicate, four ballot words of pass bits and their
//      count in shared memory;
//   2. it scans the segment counts into offsets inside the CTA and
//      publishes its per-predicate totals;
//   3. one grid barrier (all CTAs are resident: cooperative launch), after
//      which each CTA sums the totals of the CTAs before it;
//   4. it writes the ids of its passing rows from the bits, at CTA offset +
//      segment offset + rank in the segment.
// The columns are never re-read, so the traffic is the algorithmic one:
// 8 B per row plus 4 B per passing row.  A round covers as many rows as the
// bits of all CTAs hold (one round up to ~12M rows at 16 predicates).
//
// The grid barrier is a 64-bit arrival counter that is never reset: the
// host keeps its value at each launch, and the counter sits in a buffer
// cleared once.  Its wait is bounded by the global timer; a CTA that gives
// up marks the launch failed (a flag word tagged with the launch's epoch)
// and writes UINT64_MAX counts, and CTA 0 writes the real counts only
// when no CTA failed.  Nothing is read back: the counts land in device
// memory, so a batch of calls streams back to back, one launch each.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "device_util.cuh"

namespace fknn {

namespace {

constexpr int FC_THREADS = 512;
constexpr int FC_WARPS = FC_THREADS / 32;
constexpr int FC_STEP = FC_THREADS * 4;  // rows per CTA step: a float4 of each column per thread
constexpr int FC_SEG = 128;              // rows per warp segment
constexpr int FC_DEPTH = 4;              // steps in flight per warp
constexpr uint32_t FP_MAXP = 16;         // predicates per launch
constexpr size_t FC_SMEM_MAX = 100 * 1024;  // bits + offsets per CTA, so that two CTAs share an SM
constexpr int FC_SUM_UNROLL = 10;           // CTA totals in flight per lane (one pass for up to 320 CTAs)

static_assert(FC_WARPS >= (int)FP_MAXP, "one warp per predicate sums the CTA totals");

// Per predicate the closed intervals a row must fall in:
// (label lo, label hi, ts lo, ts hi).  The host turns int32(label) == v into
// the float interval of labels that truncate to v, and open predicates into
// (-inf, inf), so the device test is four float compares per row.
struct FilterPreds {
  float4 b[FP_MAXP];
};

// 4 pass bits (rows 4 * lane + c) of one predicate
__device__ __forceinline__ uint32_t pred_bits4(const float4 &b, const float4 &lab, const float4 &t) {
  auto one = [&](float l, float ts) -> uint32_t {
    return (l >= b.x && l <= b.y && ts >= b.z && ts <= b.w) ? 1u : 0u;
  };
  return one(lab.x, t.x) | (one(lab.y, t.y) << 1) | (one(lab.z, t.z) << 2) | (one(lab.w, t.w) << 3);
}

__device__ __forceinline__ uint64_t ld_volatile_u64(const uint64_t *p) { return *(const volatile uint64_t *)p; }

// Loads one step's float4 of each column for this thread (rows r .. r + 3;
// past n: zeros and valid bits cleared).
__device__ __forceinline__ void load_step(const float *__restrict__ labels, const float *__restrict__ ts, uint32_t n,
                                          uint32_t r, float4 &a, float4 &b, uint32_t &valid) {
  if (r + 4 <= n) {
    a = __ldcs(reinterpret_cast<const float4 *>(labels + r));
    b = __ldcs(reinterpret_cast<const float4 *>(ts + r));
    valid = 0xfu;
  } else {
    float la[4] = {0.f, 0.f, 0.f, 0.f}, tb[4] = {0.f, 0.f, 0.f, 0.f};
    valid = 0;
    for (int c = 0; c < 4; ++c)
      if (r + c < n) {
        la[c] = labels[r + c];
        tb[c] = ts[r + c];
        valid |= 1u << c;
      }
    a = make_float4(la[0], la[1], la[2], la[3]);
    b = make_float4(tb[0], tb[1], tb[2], tb[3]);
  }
}

// Grid: G CTAs, all resident.  Rows per CTA per round: R (a multiple of
// FC_STEP).  Dynamic shared memory: np x nseg x uint4 bits, then np x nseg
// offsets (nseg = R / FC_SEG).  sync: [0] the arrival counter (value
// bar_base at this launch), [1] the failure flag, [2 ..] 2 x G x FP_MAXP
// per-round CTA totals (double-buffered by round parity).  Row ids fit
// 32 bits (n < 2^31).
__global__ void __launch_bounds__(FC_THREADS, 2)
    k_filter_coop(const float *__restrict__ labels, const float *__restrict__ ts, uint32_t n, FilterPreds P,
                  uint32_t np, uint32_t R, uint32_t rounds, uint64_t *sync, uint64_t bar_base, uint32_t ep,
                  uint32_t *__restrict__ out, uint64_t out_stride, uint64_t *__restrict__ counts) {
  extern __shared__ __align__(16) unsigned char fc_smem[];
  const uint32_t nseg = R / FC_SEG;
  uint4 *bits = reinterpret_cast<uint4 *>(fc_smem);                           // [np][nseg]
  uint32_t *segoff = reinterpret_cast<uint32_t *>(bits + (size_t)np * nseg);  // [np][nseg]
  __shared__ float4 pb[FP_MAXP];
  __shared__ uint32_t wtot[FP_MAXP][FC_WARPS];
  __shared__ uint64_t s_off[FP_MAXP], s_base[FP_MAXP];
  __shared__ int s_fail;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t G = gridDim.x, cta = blockIdx.x;
  const uint32_t nsteps = R / FC_STEP;
  if (tid < (int)FP_MAXP) {
    pb[tid] = P.b[tid];
    s_base[tid] = 0;
  }
  __syncthreads();
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(sync);
  uint64_t *flag = sync + 1, *part = sync + 2;
  const uint32_t lanemask_lt = (1u << lane) - 1u;

  for (uint32_t rd = 0; rd < rounds; ++rd) {
    // this thread's rows of step s: row0 + s * FC_STEP + 4 * lane + c (warp w's segment s * FC_WARPS + w)
    const uint32_t row0 = (rd * G + cta) * R + w * FC_SEG + 4 * lane;
    // ---- 1. pass bits and counts per warp segment
    float4 la[FC_DEPTH], tb[FC_DEPTH];
    uint32_t vb[FC_DEPTH];
#pragma unroll
    for (int d = 0; d < FC_DEPTH; ++d)
      if ((uint32_t)d < nsteps) load_step(labels, ts, n, row0 + d * FC_STEP, la[d], tb[d], vb[d]);
    for (uint32_t s0 = 0; s0 < nsteps; s0 += FC_DEPTH) {
#pragma unroll
      for (int d = 0; d < FC_DEPTH; ++d) {
        const uint32_t s = s0 + d;
        if (s < nsteps) {
          const uint32_t seg = s * FC_WARPS + w;
          for (uint32_t p = 0; p < np; ++p) {
            const uint32_t b4 = pred_bits4(pb[p], la[d], tb[d]) & vb[d];
            const uint32_t m0 = __ballot_sync(0xffffffffu, b4 & 1u), m1 = __ballot_sync(0xffffffffu, b4 & 2u);
            const uint32_t m2 = __ballot_sync(0xffffffffu, b4 & 4u), m3 = __ballot_sync(0xffffffffu, b4 & 8u);
            if (lane == 0) {
              bits[p * nseg + seg] = make_uint4(m0, m1, m2, m3);
              segoff[p * nseg + seg] = __popc(m0) + __popc(m1) + __popc(m2) + __popc(m3);
            }
          }
          const uint32_t sn = s + FC_DEPTH;  // the step this slot carries next
          if (sn < nsteps) load_step(labels, ts, n, row0 + sn * FC_STEP, la[d], tb[d], vb[d]);
        }
      }
    }
    __syncthreads();
    // ---- 2. segment offsets inside the CTA (segments in row order), totals
    for (uint32_t i0 = 0; i0 < nseg; i0 += FC_THREADS) {
      const uint32_t i = i0 + tid;
      for (uint32_t p = 0; p < np; ++p) {
        const uint32_t v = i < nseg ? segoff[p * nseg + i] : 0u;
        uint32_t inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t x = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= o) inc += x;
        }
        if (i < nseg) segoff[p * nseg + i] = inc - v;  // exclusive within the warp's 32 segments
        if (lane == 31) wtot[p][w] = inc;
      }
      __syncthreads();
      if (tid < (int)np) {  // the warps' totals -> exclusive prefixes, carried across chunks of segments
        const uint64_t carry = i0 ? s_off[tid] : 0u;  // the running total of the earlier chunks
        uint32_t acc = (uint32_t)carry;
        for (int j = 0; j < FC_WARPS; ++j) {
          const uint32_t x = wtot[tid][j];
          wtot[tid][j] = acc;
          acc += x;
        }
        s_off[tid] = acc;
      }
      __syncthreads();
      if (i < nseg)
        for (uint32_t p = 0; p < np; ++p) segoff[p * nseg + i] += wtot[p][w];
      __syncthreads();
    }
    // the CTA's totals for this round
    uint64_t *mypart = part + ((size_t)(rd & 1) * G + cta) * FP_MAXP;
    if (tid < (int)np) {
      mypart[tid] = s_off[tid];
      __threadfence();  // visible to every CTA before this CTA arrives at the barrier
    }
    // ---- 3. grid barrier (bounded)
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      atomicAdd(bar, 1ull);
      const uint64_t target = bar_base + (uint64_t)(rd + 1) * G;
      int f = 0;
      if (ld_volatile_u64(sync) < target) {
        const uint64_t t0 = global_ns();
        while (ld_volatile_u64(sync) < target) {
          if (global_ns() - t0 > WAIT_NS) {
            f = 1;
            break;
          }
          __nanosleep(32);
        }
      }
      __threadfence();
      s_fail = f;
    }
    __syncthreads();
    if (s_fail) {
      // this launch's outputs are incomplete: flag it, poison the counts
      if (tid == 0) {
        *(volatile uint64_t *)flag = ep;
        __threadfence();
      }
      __syncthreads();
      if (tid < (int)np) counts[tid] = ~0ull;
      return;
    }
    // ---- the CTAs before this one: this CTA's offset; all: the round total
    if (w < (int)np) {
      const uint64_t *rp = part + (size_t)(rd & 1) * G * FP_MAXP;
      uint64_t before = 0, all = 0;
      for (uint32_t c0 = 0; c0 < G; c0 += 32 * FC_SUM_UNROLL) {
        uint64_t x[FC_SUM_UNROLL];
#pragma unroll
        for (int j = 0; j < FC_SUM_UNROLL; ++j) {  // the loads first, all in flight
          const uint32_t c = c0 + j * 32 + lane;
          x[j] = c < G ? __ldcg(rp + (size_t)c * FP_MAXP + w) : 0ull;
        }
#pragma unroll
        for (int j = 0; j < FC_SUM_UNROLL; ++j) {
          all += x[j];
          if (c0 + j * 32 + lane < cta) before += x[j];
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        before += __shfl_xor_sync(0xffffffffu, before, o);
        all += __shfl_xor_sync(0xffffffffu, all, o);
      }
      if (lane == 0) {
        s_off[w] = s_base[w] + before;
        s_base[w] += all;
      }
    }
    __syncthreads();
    // ---- 4. ids of the passing rows, from the bits (a segment's bits are
    // the same for the whole warp, so its skip is uniform)
    for (uint32_t p = 0; p < np; ++p) {
      uint32_t *op = out + p * out_stride;
      const uint32_t base = (uint32_t)s_off[p];
      const uint4 *bp = bits + p * nseg + w;
      const uint32_t *sp = segoff + p * nseg + w;
      for (uint32_t s = 0; s < nsteps; ++s) {
        const uint4 m = bp[s * FC_WARPS];
        if ((m.x | m.y | m.z | m.w) == 0u) continue;
        const uint32_t b4 = ((m.x >> lane) & 1u) | (((m.y >> lane) & 1u) << 1) | (((m.z >> lane) & 1u) << 2) |
                            (((m.w >> lane) & 1u) << 3);
        if (b4) {
          uint32_t pos = base + sp[s * FC_WARPS] + __popc(m.x & lanemask_lt) + __popc(m.y & lanemask_lt) +
                         __popc(m.z & lanemask_lt) + __popc(m.w & lanemask_lt);
          const uint32_t r = row0 + s * FC_STEP;
#pragma unroll
          for (int c = 0; c < 4; ++c)
            if ((b4 >> c) & 1u) op[pos++] = r + c;
        }
      }
    }
    __syncthreads();  // bits and offsets are rewritten by the next round
  }
  if (cta == 0 && tid < (int)np) {
    const bool failed = ld_volatile_u64(flag) == ep;
    counts[tid] = failed ? ~0ull : s_base[tid];
  }
}

// The floats that int32 truncation maps to v: a closed interval [lo, hi]
// (empty: lo > hi) — the label test int32(label) == v of utils.h:118 as two
// float compares.
void label_interval(int32_t v, float &lo, float &hi) {
  auto trunc_is = [v](float f) {
    const double d = std::trunc((double)f);
    return d >= -2147483648.0 && d < 2147483648.0 && (int64_t)d == (int64_t)v;
  };
  const double dv = (double)v;
  float a, b;
  if (v > 0) {
    a = (float)dv;
    if ((double)a < dv) a = std::nextafter(a, INFINITY);
    b = (float)(dv + 1.0);
    while ((double)b >= dv + 1.0) b = std::nextafter(b, -INFINITY);
  } else if (v < 0) {
    a = (float)(dv - 1.0);
    while ((double)a <= dv - 1.0) a = std::nextafter(a, INFINITY);
    b = (float)dv;
    if ((double)b > dv) b = std::nextafter(b, -INFINITY);
  } else {
    a = std::nextafter(-1.f, INFINITY);
    b = std::nextafter(1.f, -INFINITY);
  }
  if (a <= b && trunc_is(a) && trunc_is(b)) {
    lo = a;
    hi = b;
  } else {
    lo = INFINITY;
    hi = -INFINITY;
  }
}

// (type, v, l, r) -> the row intervals of FilterPreds (types checked)
float4 pred_bounds(const float *m) {
  const int type = (int)m[0];
  float4 b = make_float4(-INFINITY, INFINITY, -INFINITY, INFINITY);
  if (type == 1 || type == 3) label_interval((int32_t)m[1], b.x, b.y);
  if (type == 2 || type == 3) {
    b.z = m[2];  // NaN bounds pass no row, as the reference's compares
    b.w = m[3];
  }
  return b;
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
  FilterState &fs = idx->filter_state;
  // resident CTAs of the cooperative grid (two per SM when the shared memory allows)
  if (!fs.grid) {
    FKNN_CUDA(cudaFuncSetAttribute(k_filter_coop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FC_SMEM_MAX));
    int per_sm = 0;
    FKNN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_filter_coop, FC_THREADS, FC_SMEM_MAX));
    if (per_sm < 1) {
      set_error("fknn_filter_rows: the compaction kernel does not fit an SM");
      return FKNN_ECUDA;
    }
    fs.grid = (uint32_t)idx->num_sms * (uint32_t)std::min(per_sm, 2);
  }
  const uint32_t G = fs.grid;
  // sync words: arrival counter, failure flag, 2 x G x FP_MAXP CTA totals;
  // cleared when the buffer is new or the epochs run out
  const size_t words = 2 + 2 * (size_t)G * FP_MAXP;
  uint64_t *sync;
  int rc;
  if ((rc = ws_get(idx, 16, words * sizeof(uint64_t), (void **)&sync))) return rc;
  if (fs.status != sync || fs.bytes != idx->ws[16].bytes || fs.epoch >= (1u << 30)) {
    FKNN_CUDA(cudaMemsetAsync(sync, 0, words * sizeof(uint64_t), st));
    fs.status = sync;
    fs.bytes = idx->ws[16].bytes;
    fs.epoch = 0;
    fs.arrivals = 0;
  }
  for (uint32_t p0 = 0; p0 < np; p0 += FP_MAXP) {
    const uint32_t m = std::min<uint32_t>(FP_MAXP, np - p0);
    // rows per CTA per round: as few rounds as the bits allow, rows split evenly
    const size_t per_row = (size_t)m * (sizeof(uint4) + sizeof(uint32_t));  // per 128-row segment
    const uint64_t r_cap = std::max<uint64_t>(FC_STEP, (FC_SMEM_MAX / per_row) * FC_SEG / FC_STEP * FC_STEP);
    const uint64_t rounds = std::max<uint64_t>(1, (n + (uint64_t)G * r_cap - 1) / ((uint64_t)G * r_cap));
    const uint64_t per_cta = (n + (uint64_t)G * rounds - 1) / ((uint64_t)G * rounds);
    const uint32_t R = (uint32_t)std::max<uint64_t>(FC_STEP, (per_cta + FC_STEP - 1) / FC_STEP * FC_STEP);
    const size_t smem = (size_t)(R / FC_SEG) * per_row;
    FilterPreds P;
    std::memset(&P, 0, sizeof(P));
    for (uint32_t p = 0; p < m; ++p) {
      const float *q = metas + (size_t)(p0 + p) * 4;
      P.b[p] = pred_bounds(q);
    }
    const float *lab = idx->labels_f, *tsv = idx->ts_f;
    uint32_t nn = (uint32_t)n;
    uint64_t bar_base = fs.arrivals, stride = n;
    uint32_t mm = m, RR = R, nr = (uint32_t)rounds, ep = ++fs.epoch;
    uint32_t *o = d_out + (uint64_t)p0 * n;
    uint64_t *c = d_counts + p0;
    void *args[] = {(void *)&lab, (void *)&tsv, (void *)&nn, (void *)&P, (void *)&mm, (void *)&RR, (void *)&nr,
                    (void *)&sync, (void *)&bar_base, (void *)&ep, (void *)&o, (void *)&stride, (void *)&c};
    FKNN_CUDA(cudaLaunchCooperativeKernel((const void *)k_filter_coop, dim3(G), dim3(FC_THREADS), args, smem, st));
    fs.arrivals += rounds * G;
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
