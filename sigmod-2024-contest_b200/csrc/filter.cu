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
constexpr int FC_SEG = 128;                        // rows per segment: one set of four ballot words
constexpr int FC_SEGS = 2;                         // segments per warp in a tile
constexpr int FC_TSEG = FC_WARPS * FC_SEGS;        // segments per tile (32)
constexpr int FC_TILE = FC_TSEG * FC_SEG;          // rows per tile (4,096)
constexpr uint32_t FP_MAXP = 16;                   // predicates per launch
constexpr uint32_t FC_STAGE_BYTES = 2 * FC_TILE * 4;  // one ring stage: a tile of both columns (32 KB)
constexpr uint32_t FC_SMAX = 3;                    // ring stages at most
constexpr uint32_t FC_LAG = 2;                     // rows between a tile's count and its ids
constexpr uint32_t FC_SLOTS = FC_LAG + 2;          // bits slots (the writer's, the counter's and one between)
constexpr size_t FC_SMEM_MAX = 108 * 1024;         // dynamic shared memory per CTA: two CTAs share an SM
constexpr int FC_SUM_UNROLL = 10;                  // tile counts per lane of a row (rows of up to 320 CTAs)

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

// Grid: G CTAs, all resident (cooperative launch).  Tiles of FC_TILE rows in
// row order; CTA c takes tiles j * G + c, j = 0 .. nrow - 1 ("row" j of
// tiles).  At step j a CTA counts its tile of row j (bits and counts kept
// in a shared-memory slot, its tile count published), and writes the ids of
// its tile of row j - FC_LAG, whose place is the counts of all tiles before
// it: the rows before (a running total) plus the CTAs before it in its row.
// Those counts were published FC_LAG steps earlier, so the ids stream out
// while the columns stream in.  Dynamic shared memory: S ring stages of
// FC_TILE rows of both columns (bulk copies), FC_SLOTS slots of np x
// FC_TSEG bits and segment offsets, a 128-id staging slice per warp.
// agg: nrow x G x FP_MAXP words (epoch tag << 16 | tile count); flag: the
// failure flag (tagged with ep).  Row ids fit 32 bits (n < 2^31).
__global__ void __launch_bounds__(FC_THREADS, 2)
    k_filter_coop(const float *__restrict__ labels, const float *__restrict__ ts, uint32_t n, FilterPreds P,
                  uint32_t np, uint32_t nrow, uint32_t S, uint32_t *agg, uint64_t *flag, uint32_t ep,
                  uint32_t *__restrict__ out, uint64_t out_stride, uint64_t *__restrict__ counts, int *err) {
  extern __shared__ __align__(128) unsigned char fc_smem[];
  float *ring = reinterpret_cast<float *>(fc_smem);  // stage st: labels [FC_TILE], ts [FC_TILE]
  uint4 *bits = reinterpret_cast<uint4 *>(fc_smem + (size_t)S * FC_STAGE_BYTES);   // [slot][np][FC_TSEG]
  uint32_t *segx = reinterpret_cast<uint32_t *>(bits + (size_t)FC_SLOTS * np * FC_TSEG);  // same shape
  uint32_t *stage_all = segx + (size_t)FC_SLOTS * np * FC_TSEG;                     // [warp][FC_SEG]
  __shared__ uint64_t full[FC_SMAX];
  __shared__ float4 pb[FP_MAXP];
  __shared__ uint32_t s_pref[FP_MAXP];
  __shared__ uint64_t s_rowbase[FP_MAXP];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t G = gridDim.x, cta = blockIdx.x;
  const uint32_t tag = (ep & 0xffffu) << 16;
  if (tid < (int)FP_MAXP) {
    pb[tid] = P.b[tid];
    s_rowbase[tid] = 0;
  }
  if (tid == 0) {
    for (uint32_t st = 0; st < S; ++st) mbar_init(&full[st], 1);
    fence_mbar_init();
  }
  __syncthreads();
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  auto tile_full = [&](uint32_t t) { return (uint64_t)(t + 1) * FC_TILE <= n; };
  auto issue = [&](uint32_t t, uint32_t st) {
    float *dst = ring + st * (2 * FC_TILE);
    mbar_arrive_expect_tx(&full[st], FC_STAGE_BYTES);
    bulk_g2s(dst, labels + (size_t)t * FC_TILE, FC_TILE * 4, &full[st]);
    bulk_g2s(dst + FC_TILE, ts + (size_t)t * FC_TILE, FC_TILE * 4, &full[st]);
  };
  uint32_t pend = 0;  // bit st: a copy into stage st is in flight (the same in every thread)
  for (uint32_t j = 0; j < S && j < nrow; ++j)
    if (tile_full(j * G + cta)) {
      if (tid == 0) issue(j * G + cta, j);
      pend |= 1u << j;
    }
  uint32_t phase = 0;         // bit st: the parity of stage st's next completion (the same in every thread)
  uint32_t st = 0;            // ring stage of row j (j mod S)
  uint32_t slot = 0;          // bits slot of row j (j mod FC_SLOTS)
  uint32_t *stage = stage_all + w * FC_SEG;
  bool failed = false;
  for (uint32_t j = 0; j < nrow + FC_LAG; ++j) {
    const bool counting = j < nrow, writing = j >= FC_LAG;
    const uint32_t jw = j - FC_LAG, wslot = (slot + FC_SLOTS - FC_LAG) % FC_SLOTS;
    // the counts of row jw, loaded early (published FC_LAG steps ago)
    uint32_t x[FC_SUM_UNROLL];
    if (writing && w < (int)np) {
#pragma unroll
      for (int k = 0; k < FC_SUM_UNROLL; ++k) {
        const uint32_t c2 = k * 32 + lane;
        x[k] = c2 < G ? ld_volatile_u32(agg + ((size_t)jw * G + c2) * FP_MAXP + w) : tag;
      }
    }
    // ---- count the tile of row j
    if (counting) {
      const uint32_t t = j * G + cta;
      float4 la[FC_SEGS], tb[FC_SEGS];
      uint32_t vb[FC_SEGS];
      if (tile_full(t)) {
        // warp-uniform: the lanes' timers may disagree at the deadline
        if (__all_sync(0xffffffffu, mbar_wait_bounded(&full[st], (phase >> st) & 1u, err))) {
          phase ^= 1u << st;
          pend &= ~(1u << st);
        } else {
          failed = true;  // the copy is still pending, at the same parity
        }
        const float *src = ring + st * (2 * FC_TILE) + w * (FC_SEGS * FC_SEG) + 4 * lane;
#pragma unroll
        for (int sg = 0; sg < FC_SEGS; ++sg) {
          la[sg] = *reinterpret_cast<const float4 *>(src + sg * FC_SEG);
          tb[sg] = *reinterpret_cast<const float4 *>(src + sg * FC_SEG + FC_TILE);
          vb[sg] = 0xfu;
        }
      } else {
#pragma unroll
        for (int sg = 0; sg < FC_SEGS; ++sg)
          load_step(labels, ts, n, t * FC_TILE + w * (FC_SEGS * FC_SEG) + sg * FC_SEG + 4 * lane, la[sg], tb[sg],
                    vb[sg]);
      }
      for (uint32_t p = 0; p < np; ++p) {
#pragma unroll
        for (int sg = 0; sg < FC_SEGS; ++sg) {
          const uint32_t b4 = pred_bits4(pb[p], la[sg], tb[sg]) & vb[sg];
          const uint32_t m0 = __ballot_sync(0xffffffffu, b4 & 1u), m1 = __ballot_sync(0xffffffffu, b4 & 2u);
          const uint32_t m2 = __ballot_sync(0xffffffffu, b4 & 4u), m3 = __ballot_sync(0xffffffffu, b4 & 8u);
          if (lane == 0) {
            const uint32_t i = (slot * np + p) * FC_TSEG + w * FC_SEGS + sg;
            bits[i] = make_uint4(m0, m1, m2, m3);
            segx[i] = __popc(m0) + __popc(m1) + __popc(m2) + __popc(m3);
          }
        }
      }
    }
    if (__syncthreads_or(failed)) {
      failed = true;
      break;
    }
    if (counting) {
      if (tid < (int)np) {
        // segment offsets inside the tile; the tile's count, published
        uint32_t *sx = segx + (slot * np + tid) * FC_TSEG, acc = 0;
        for (int i = 0; i < FC_TSEG; ++i) {
          const uint32_t v = sx[i];
          sx[i] = acc;
          acc += v;
        }
        *(volatile uint32_t *)(agg + ((size_t)j * G + cta) * FP_MAXP + tid) = tag | acc;
      }
      // the stage of row j is free (every warp is past the barrier): refill it
      if (j + S < nrow && tile_full((j + S) * G + cta)) {
        if (tid == 0) issue((j + S) * G + cta, st);
        pend |= 1u << st;
      }
      if (++st == S) st = 0;
    }
    // ---- the place of this CTA's tile of row jw
    if (writing && w < (int)np) {
      const uint64_t t0 = global_ns();
      bool ok = true;
#pragma unroll
      for (int k = 0; k < FC_SUM_UNROLL; ++k) {
        const uint32_t c2 = k * 32 + lane;
        while (ok && (x[k] & 0xffff0000u) != tag) {
          if (global_ns() - t0 > WAIT_NS) ok = false;
          else x[k] = ld_volatile_u32(agg + ((size_t)jw * G + c2) * FP_MAXP + w);
        }
      }
      uint32_t before = 0, all = 0;
#pragma unroll
      for (int k = 0; k < FC_SUM_UNROLL; ++k) {
        const uint32_t c2 = k * 32 + lane, v = c2 < G ? (x[k] & 0xffffu) : 0u;
        all += v;
        if (c2 < cta) before += v;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        before += __shfl_xor_sync(0xffffffffu, before, o);
        all += __shfl_xor_sync(0xffffffffu, all, o);
      }
      if (!__all_sync(0xffffffffu, ok)) failed = true;
      if (lane == 0) {
        s_pref[w] = (uint32_t)s_rowbase[w] + before;
        s_rowbase[w] += all;
      }
    }
    if (__syncthreads_or(failed)) {
      failed = true;
      break;
    }
    // ---- its ids, staged per segment and stored contiguously
    if (writing) {
      const uint32_t tw = jw * G + cta;
      for (uint32_t p = 0; p < np; ++p) {
        uint32_t *op = out + p * out_stride;
#pragma unroll
        for (int sg = 0; sg < FC_SEGS; ++sg) {
          const uint32_t i = (wslot * np + p) * FC_TSEG + w * FC_SEGS + sg;
          const uint4 m = bits[i];  // the same for the whole warp: the skip is uniform
          const uint32_t cnt = __popc(m.x) + __popc(m.y) + __popc(m.z) + __popc(m.w);
          if (cnt == 0) continue;
          const uint32_t b4 = ((m.x >> lane) & 1u) | (((m.y >> lane) & 1u) << 1) | (((m.z >> lane) & 1u) << 2) |
                              (((m.w >> lane) & 1u) << 3);
          uint32_t k = __popc(m.x & lanemask_lt) + __popc(m.y & lanemask_lt) + __popc(m.z & lanemask_lt) +
                       __popc(m.w & lanemask_lt);
          const uint32_t r = tw * FC_TILE + w * (FC_SEGS * FC_SEG) + sg * FC_SEG + 4 * lane;
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if ((b4 >> q) & 1u) stage[k++] = r + q;
          __syncwarp();
          uint32_t *dst = op + s_pref[p] + segx[i];
          for (uint32_t jj = lane; jj < cnt; jj += 32) dst[jj] = stage[jj];
          __syncwarp();  // the slice is rewritten by the next segment
        }
      }
    }
    if (++slot == FC_SLOTS) slot = 0;
  }
  if (failed) {
    // a wait gave up: wait (bounded) for this CTA's copies still in flight,
    // flag the launch and poison the counts
    if (tid == 0) {
      for (uint32_t s2 = 0; s2 < S; ++s2)
        if ((pend >> s2) & 1u) mbar_wait_bounded(&full[s2], (phase >> s2) & 1u, err);
      *(volatile uint64_t *)flag = ep;
      __threadfence();
    }
    __syncthreads();
    if (tid < (int)np) counts[tid] = ~0ull;
    return;
  }
  if (cta == 0 && tid < (int)np) {
    __threadfence();
    const bool bad = ld_volatile_u64(flag) == ep;
    counts[tid] = bad ? ~0ull : s_rowbase[tid];
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
    fs.grid = std::min<uint32_t>((uint32_t)idx->num_sms * (uint32_t)std::min(per_sm, 2), 32 * FC_SUM_UNROLL);
  }
  const uint32_t G = fs.grid;
  const uint32_t ntiles = (uint32_t)((n + FC_TILE - 1) / FC_TILE), nrow = (ntiles + G - 1) / G;
  // the failure flag, then nrow x G x FP_MAXP tagged tile counts; cleared
  // when the buffer is new or the 16-bit epochs run out
  const size_t bytes = 64 + (size_t)nrow * G * FP_MAXP * 4;
  unsigned char *sync;
  int rc;
  if ((rc = ws_get(idx, 16, bytes, (void **)&sync))) return rc;
  if (fs.status != sync || fs.bytes != idx->ws[16].bytes || fs.epoch >= 0xffffu) {
    FKNN_CUDA(cudaMemsetAsync(sync, 0, bytes, st));
    fs.status = sync;
    fs.bytes = idx->ws[16].bytes;
    fs.epoch = 0;
  }
  for (uint32_t p0 = 0; p0 < np; p0 += FP_MAXP) {
    const uint32_t m = std::min<uint32_t>(FP_MAXP, np - p0);
    // shared memory: the bits slots, the staging slices, and as many ring
    // stages as fit (at least one)
    const size_t slots = (size_t)FC_SLOTS * m * FC_TSEG * (sizeof(uint4) + sizeof(uint32_t));
    const size_t staging = (size_t)FC_WARPS * FC_SEG * sizeof(uint32_t);
    const uint32_t S = (uint32_t)std::max<size_t>(
        1, std::min<size_t>(FC_SMAX, (FC_SMEM_MAX - slots - staging) / FC_STAGE_BYTES));
    const size_t smem = (size_t)S * FC_STAGE_BYTES + slots + staging;
    FilterPreds P;
    std::memset(&P, 0, sizeof(P));
    for (uint32_t p = 0; p < m; ++p) P.b[p] = pred_bounds(metas + (size_t)(p0 + p) * 4);
    const float *lab = idx->labels_f, *tsv = idx->ts_f;
    uint32_t nn = (uint32_t)n, mm = m, nr = nrow, SS = S, ep = ++fs.epoch;
    uint32_t *agg = reinterpret_cast<uint32_t *>(sync + 64);
    uint64_t *flag = reinterpret_cast<uint64_t *>(sync);
    uint64_t stride = n;
    uint32_t *o = d_out + (uint64_t)p0 * n;
    uint64_t *c = d_counts + p0;
    int *errp = idx->d_flag;
    void *args[] = {(void *)&lab,  (void *)&tsv, (void *)&nn,     (void *)&P, (void *)&mm,
                    (void *)&nr,   (void *)&SS,  (void *)&agg,    (void *)&flag, (void *)&ep,
                    (void *)&o,    (void *)&stride, (void *)&c,   (void *)&errp};
    FKNN_CUDA(cudaLaunchCooperativeKernel((const void *)k_filter_coop, dim3(G), dim3(FC_THREADS), args, smem, st));
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
