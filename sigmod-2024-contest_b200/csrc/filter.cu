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
constexpr uint32_t FP_MAXP = 16;         // predicates per launch
constexpr size_t FC_SMEM_MAX = 104 * 1024;  // ring + bits + offsets per CTA, so that two CTAs share an SM
constexpr uint32_t FC_STAGE_BYTES = 2 * FC_STEP * 4;  // one ring stage: FC_STEP rows of both columns
constexpr uint32_t FC_SMAX = 6;                      // ring stages at most
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
// FC_STEP).  Dynamic shared memory: S ring stages of FC_STEP rows of both
// columns (bulk copies), then np x nseg x uint4 bits and np x nseg segment
// offsets (nseg = R / FC_SEG).  sync: [0] the arrival counter (value
// bar_base at this launch), [1] the failure flag, [2 ..] 2 x G x FP_MAXP
// per-round CTA totals (double-buffered by round parity).  Row ids fit
// 32 bits (n < 2^31).
__global__ void __launch_bounds__(FC_THREADS, 2)
    k_filter_coop(const float *__restrict__ labels, const float *__restrict__ ts, uint32_t n, FilterPreds P,
                  uint32_t np, uint32_t R, uint32_t rounds, uint32_t S, uint64_t *sync, uint64_t bar_base,
                  uint32_t ep, uint32_t *__restrict__ out, uint64_t out_stride, uint64_t *__restrict__ counts,
                  int *err) {
  extern __shared__ __align__(128) unsigned char fc_smem[];
  const uint32_t nseg = R / FC_SEG, nchunk = R / FC_STEP;
  float *ring = reinterpret_cast<float *>(fc_smem);  // stage st: labels [FC_STEP], ts [FC_STEP]
  uint4 *bits = reinterpret_cast<uint4 *>(fc_smem + (size_t)S * FC_STAGE_BYTES);  // [np][nseg]
  uint32_t *segoff = reinterpret_cast<uint32_t *>(bits + (size_t)np * nseg);      // [np][nseg]
  __shared__ uint64_t full[FC_SMAX];
  __shared__ float4 pb[FP_MAXP];
  __shared__ uint32_t wtot[FP_MAXP][FC_WARPS], wsum[FP_MAXP][FC_WARPS];
  __shared__ uint64_t s_off[FP_MAXP], s_base[FP_MAXP];
  __shared__ int s_fail;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t G = gridDim.x, cta = blockIdx.x;
  if (tid < (int)FP_MAXP) {
    pb[tid] = P.b[tid];
    s_base[tid] = 0;
  }
  if (tid == 0) {
    for (uint32_t st = 0; st < S; ++st) mbar_init(&full[st], 1);
    fence_mbar_init();
  }
  __syncthreads();
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(sync);
  uint64_t *flag = sync + 1, *part = sync + 2;
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  uint32_t phase = 0;  // bit st: the parity of stage st's next completion (the same in every thread)

  for (uint32_t rd = 0; rd < rounds; ++rd) {
    const uint32_t cbase = (rd * G + cta) * R;  // the CTA's first row this round
    // chunks 0 .. nfull-1 have all their rows and are copied in bulk; the
    // (one) partial chunk of the base is read by the threads themselves
    const uint32_t nfull = n > cbase ? min(nchunk, (n - cbase) / FC_STEP) : 0u;
    auto issue = [&](uint32_t c, uint32_t st) {
      float *dst = ring + st * (2 * FC_STEP);
      mbar_arrive_expect_tx(&full[st], FC_STAGE_BYTES);
      bulk_g2s(dst, labels + cbase + c * FC_STEP, FC_STEP * 4, &full[st]);
      bulk_g2s(dst + FC_STEP, ts + cbase + c * FC_STEP, FC_STEP * 4, &full[st]);
    };
    if (tid == 0)
      for (uint32_t c = 0; c < S && c < nfull; ++c) issue(c, c);
    for (uint32_t p = tid; p < np * FC_WARPS; p += FC_THREADS) wsum[p / FC_WARPS][p % FC_WARPS] = 0;
    __syncthreads();
    // ---- 1. pass bits per warp segment (segment c * FC_WARPS + w: rows
    //         cbase + c * FC_STEP + w * FC_SEG + 4 * lane + 0..3)
    bool gave_up = false;
    uint32_t c = 0, st = 0;  // chunk, its ring stage (c mod S)
    const float *mine = ring + w * FC_SEG + 4 * lane;
    for (; c < nchunk; ++c) {
      const uint32_t seg = c * FC_WARPS + w;
      float4 la, tb;
      uint32_t vb = 0xfu;
      if (c < nfull) {
        // warp-uniform: the lanes' timers may disagree at the deadline
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full[st], (phase >> st) & 1u, err))) gave_up = true;
        phase ^= 1u << st;
        la = *reinterpret_cast<const float4 *>(mine + st * (2 * FC_STEP));
        tb = *reinterpret_cast<const float4 *>(mine + st * (2 * FC_STEP) + FC_STEP);
      } else {
        load_step(labels, ts, n, cbase + c * FC_STEP + w * FC_SEG + 4 * lane, la, tb, vb);
      }
      for (uint32_t p = 0; p < np; ++p) {
        const uint32_t b4 = pred_bits4(pb[p], la, tb) & vb;
        const uint32_t m0 = __ballot_sync(0xffffffffu, b4 & 1u), m1 = __ballot_sync(0xffffffffu, b4 & 2u);
        const uint32_t m2 = __ballot_sync(0xffffffffu, b4 & 4u), m3 = __ballot_sync(0xffffffffu, b4 & 8u);
        if (lane == 0) {
          const uint32_t cnt = __popc(m0) + __popc(m1) + __popc(m2) + __popc(m3);
          bits[p * nseg + seg] = make_uint4(m0, m1, m2, m3);
          segoff[p * nseg + seg] = cnt;
          wsum[p][w] += cnt;
        }
      }
      // the stage is free once every warp has read it; refill it
      if (__syncthreads_or(gave_up)) {
        gave_up = true;
        break;
      }
      if (tid == 0 && c + S < nfull) issue(c + S, st);
      if (++st == S) st = 0;
    }
    if (gave_up) {
      // a copy did not land in time: wait (bounded) for this CTA's copies
      // still in flight, flag the launch and poison the counts
      if (tid == 0) {
        uint32_t st2 = st;
        for (uint32_t c2 = c; c2 < c + S && c2 < nfull; ++c2) {
          const uint32_t par = c2 == c ? (((phase >> st2) & 1u) ^ 1u) : ((phase >> st2) & 1u);
          mbar_wait_bounded(&full[st2], par, err);
          if (++st2 == S) st2 = 0;
        }
        *(volatile uint64_t *)flag = ep;
        __threadfence();
      }
      __syncthreads();
      if (tid < (int)np) counts[tid] = ~0ull;
      return;
    }
    // ---- 2. the CTA's totals, published; the barrier arrival (release)
    if (tid == 0) {
      uint64_t *mypart = part + ((size_t)(rd & 1) * G + cta) * FP_MAXP;
      for (uint32_t p = 0; p < np; ++p) {
        uint32_t t = 0;
        for (int j = 0; j < FC_WARPS; ++j) t += wsum[p][j];
        mypart[p] = t;
      }
      asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(bar), "l"(1ull) : "memory");
    }
    // ---- 3. segment offsets inside the CTA, while the other CTAs finish
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
        uint32_t acc = i0 ? (uint32_t)s_off[tid] : 0u;  // the running total of the earlier chunks
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
    // ---- 4. the grid barrier's wait (bounded, acquire)
    if (tid == 0) {
      const uint64_t target = bar_base + (uint64_t)(rd + 1) * G;
      auto now = [&]() {
        uint64_t v;
        asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(bar) : "memory");
        return v;
      };
      int f = 0;
      if (now() < target) {
        const uint64_t t0 = global_ns();
        while (now() < target) {
          if (global_ns() - t0 > WAIT_NS) {
            f = 1;
            break;
          }
        }
      }
      s_fail = f;
    }
    __syncthreads();
    if (s_fail) {
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
          const uint32_t cc = c0 + j * 32 + lane;
          x[j] = cc < G ? __ldcg(rp + (size_t)cc * FP_MAXP + w) : 0ull;
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
    // ---- 5. ids of the passing rows: per segment staged in this warp's
    //         slice of the (now idle) ring, then stored contiguously
    uint32_t *stage = reinterpret_cast<uint32_t *>(ring) + w * FC_SEG;
    for (uint32_t p = 0; p < np; ++p) {
      uint32_t *op = out + p * out_stride;
      const uint32_t base = (uint32_t)s_off[p];
      const uint4 *bp = bits + p * nseg + w;
      const uint32_t *sp = segoff + p * nseg + w;
      for (uint32_t cc = 0; cc < nchunk; ++cc) {
        const uint4 m = bp[cc * FC_WARPS];  // the same for the whole warp: the skip is uniform
        const uint32_t cnt = __popc(m.x) + __popc(m.y) + __popc(m.z) + __popc(m.w);
        if (cnt == 0) continue;
        const uint32_t b4 = ((m.x >> lane) & 1u) | (((m.y >> lane) & 1u) << 1) | (((m.z >> lane) & 1u) << 2) |
                            (((m.w >> lane) & 1u) << 3);
        uint32_t k = __popc(m.x & lanemask_lt) + __popc(m.y & lanemask_lt) + __popc(m.z & lanemask_lt) +
                     __popc(m.w & lanemask_lt);
        const uint32_t r = cbase + cc * FC_STEP + w * FC_SEG + 4 * lane;
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if ((b4 >> q) & 1u) stage[k++] = r + q;
        __syncwarp();
        uint32_t *dst = op + base + sp[cc * FC_WARPS];
        for (uint32_t j = lane; j < cnt; j += 32) dst[j] = stage[j];
        __syncwarp();  // the slice is rewritten by the next segment
      }
    }
    // the ring's generic writes before the next round's bulk copies into it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();  // bits, offsets and the ring are rewritten by the next round
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
    // rows per CTA per round and ring stages: one round with the deepest
    // ring the shared memory leaves room for, else two stages and as few
    // rounds as the bits allow (rows split evenly)
    const size_t per_seg = (size_t)m * (sizeof(uint4) + sizeof(uint32_t));  // bits + offset per 128 rows
    const uint64_t one = ((n + G - 1) / G + FC_STEP - 1) / FC_STEP * FC_STEP;
    uint32_t S;
    uint64_t rounds, R;
    if ((one / FC_SEG) * per_seg + 2 * FC_STAGE_BYTES <= FC_SMEM_MAX) {
      rounds = 1;
      R = one;
      S = (uint32_t)std::min<size_t>(FC_SMAX, (FC_SMEM_MAX - (one / FC_SEG) * per_seg) / FC_STAGE_BYTES);
    } else {
      S = 2;
      const uint64_t r_cap = std::max<uint64_t>(
          FC_STEP, ((FC_SMEM_MAX - 2 * FC_STAGE_BYTES) / per_seg) * FC_SEG / FC_STEP * FC_STEP);
      rounds = (n + G * r_cap - 1) / (G * r_cap);
      const uint64_t per_cta = (n + G * rounds - 1) / (G * rounds);
      R = std::max<uint64_t>(FC_STEP, (per_cta + FC_STEP - 1) / FC_STEP * FC_STEP);
    }
    const size_t smem = (size_t)S * FC_STAGE_BYTES + (size_t)(R / FC_SEG) * per_seg;
    FilterPreds P;
    std::memset(&P, 0, sizeof(P));
    for (uint32_t p = 0; p < m; ++p) {
      const float *q = metas + (size_t)(p0 + p) * 4;
      P.b[p] = pred_bounds(q);
    }
    const float *lab = idx->labels_f, *tsv = idx->ts_f;
    uint32_t nn = (uint32_t)n;
    uint64_t bar_base = fs.arrivals, stride = n;
    uint32_t mm = m, RR = (uint32_t)R, nr = (uint32_t)rounds, SS = S, ep = ++fs.epoch;
    uint32_t *o = d_out + (uint64_t)p0 * n;
    uint64_t *c = d_counts + p0;
    int *errp = idx->d_flag;
    void *args[] = {(void *)&lab, (void *)&tsv, (void *)&nn, (void *)&P, (void *)&mm, (void *)&RR, (void *)&nr,
                    (void *)&SS, (void *)&sync, (void *)&bar_base, (void *)&ep, (void *)&o, (void *)&stride,
                    (void *)&c, (void *)&errp};
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
