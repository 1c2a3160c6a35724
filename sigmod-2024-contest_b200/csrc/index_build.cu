// Resident index construction: validation, the two row orders the
// predicates resolve to contiguous slabs in, and the blocked HBM layout the
// contraction streams.
//
// Orders (the B200 counterpart of the host sorts of utils.h:403-434 and
// hybrid_graph.cpp:505-524):
//   ORDER_TIME: rows by (ts, id)          -> type 0 (all) and type 2 (window)
//   ORDER_CAT : rows by (label, ts, id)   -> type 1 (label slab), type 3 (window in it)
// Both are produced by a stable LSD radix sort whose scatter pass is a
// warp match/ballot + prefix-sum partition (rs_scatter below).
#include "fknn_internal.cuh"

namespace fknn {

namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // 4096 keys per tile
constexpr int RS_BITS = 8;
constexpr int RS_DIGITS = 1 << RS_BITS;

__global__ void rs_hist(const uint32_t *__restrict__ keys, uint64_t n, int shift, uint32_t *__restrict__ hist,
                        uint32_t ntiles) {
  __shared__ uint32_t cnt[RS_DIGITS];
  const uint32_t tile = blockIdx.x;
  for (int d = threadIdx.x; d < RS_DIGITS; d += blockDim.x) cnt[d] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)tile * RS_TILE;
#pragma unroll 4
  for (int i = 0; i < RS_ITEMS; ++i) {
    uint64_t idx = base + (uint64_t)i * RS_THREADS + threadIdx.x;
    if (idx < n) atomicAdd(&cnt[(keys[idx] >> shift) & (RS_DIGITS - 1)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < RS_DIGITS; d += blockDim.x) hist[(uint64_t)d * ntiles + tile] = cnt[d];
}

// Exclusive scan of len counters in one block (len <= a few million).
__global__ void rs_scan(uint32_t *__restrict__ data, uint64_t len) {
  __shared__ uint32_t part[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const uint64_t per = (len + T - 1) / T;
  const uint64_t b = (uint64_t)t * per, e = b + per < len ? b + per : len;
  uint32_t s = 0;
  for (uint64_t i = b; i < e; ++i) s += data[i];
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < T; off <<= 1) {
    uint32_t v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  uint32_t run = t ? part[t - 1] : 0;
  for (uint64_t i = b; i < e; ++i) {
    uint32_t v = data[i];
    data[i] = run;
    run += v;
  }
}

// Stable scatter: rounds of 256 consecutive keys; inside a warp the rank of
// a key among equal digits comes from __match_any_sync + popc, across the
// block's warps from a per-round digit prefix in shared memory.
__global__ void rs_scatter(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                           uint32_t *__restrict__ kout, uint32_t *__restrict__ vout, uint64_t n, int shift,
                           const uint32_t *__restrict__ hist, uint32_t ntiles) {
  constexpr int NW = RS_THREADS / 32;
  __shared__ uint32_t off[RS_DIGITS];
  __shared__ uint32_t wcnt[NW][RS_DIGITS + 1];
  const uint32_t tile = blockIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < RS_DIGITS; d += blockDim.x) off[d] = hist[(uint64_t)d * ntiles + tile];
  const uint64_t base = (uint64_t)tile * RS_TILE;
  const uint32_t lt_mask = (1u << lane) - 1u;
  for (int r = 0; r < RS_ITEMS; ++r) {
    for (int i = threadIdx.x; i < NW * (RS_DIGITS + 1); i += blockDim.x) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint64_t idx = base + (uint64_t)r * RS_THREADS + threadIdx.x;
    const bool valid = idx < n;
    uint32_t key = 0, val = 0;
    int d = RS_DIGITS;  // invalid items take a private digit
    if (valid) {
      key = kin[idx];
      val = vin[idx];
      d = (key >> shift) & (RS_DIGITS - 1);
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & lt_mask);
    if (rank == 0) wcnt[w][d] = __popc(peers);
    __syncthreads();
    for (int dd = threadIdx.x; dd < RS_DIGITS; dd += blockDim.x) {
      uint32_t p = off[dd];
#pragma unroll
      for (int ww = 0; ww < NW; ++ww) {
        uint32_t c = wcnt[ww][dd];
        wcnt[ww][dd] = p;
        p += c;
      }
      off[dd] = p;
    }
    __syncthreads();
    if (valid) {
      const uint32_t pos = wcnt[w][d] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
  }
}

__global__ void k_validate_base(const float *__restrict__ vecs, const float *__restrict__ labels,
                                const float *__restrict__ ts, uint64_t n, int *flag) {
  const uint64_t total = n * DIM;
  int bad = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    float x = vecs[i];
    if (!(fabsf(x) <= 1e15f)) bad |= 1;  // also catches NaN
    if (i < n) {
      float l = labels[i], t = ts[i];
      if (!(fabsf(l) < 2147483648.f)) bad |= 2;
      if (!(fabsf(t) <= 3.0e38f)) bad |= 4;
    }
  }
  if (bad) atomicOr(flag, bad);
}

// ||x||^2 as a float FMA chain in dimension order (the same chain the
// contraction uses for q.x, so the screening bound applies).
__global__ void k_norms(const float *__restrict__ vecs, uint64_t n, float *__restrict__ norms) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float *x = vecs + i * DIM;
  float s = 0.f;
#pragma unroll 10
  for (int d = 0; d < DIM; ++d) s = fmaf(x[d], x[d], s);
  norms[i] = s;
}

__global__ void k_time_keys(const float *__restrict__ ts, uint64_t n, uint32_t *__restrict__ keys,
                            uint32_t *__restrict__ vals) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float t = ts[i];
  if (t == 0.f) t = 0.f;  // -0 sorts with +0: the predicate compares them equal
  keys[i] = f32_sortable(t);
  vals[i] = (uint32_t)i;
}

__global__ void k_label_keys(const float *__restrict__ labels, const uint32_t *__restrict__ perm, uint64_t n,
                             uint32_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t id = perm[i];
  keys[i] = i32_sortable((int32_t)labels[id]);  // float -> int32 truncation, utils.h:109
  vals[i] = id;
}

__global__ void k_order_columns(const uint32_t *__restrict__ perm, const float *__restrict__ ts,
                                const float *__restrict__ labels, uint64_t n, float *__restrict__ ts_o,
                                int32_t *__restrict__ label_o) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t id = perm[i];
  ts_o[i] = ts[id];
  label_o[i] = (int32_t)labels[id];
}

// One CTA per 64-row block: gather rows perm[b*64 .. b*64+63] (row-major,
// coalesced per row), transpose through shared memory, write [101][64].
__global__ void k_build_blocks(const float *__restrict__ vecs, const float *__restrict__ norms,
                               const uint32_t *__restrict__ perm, uint64_t n, float *__restrict__ blocks) {
  __shared__ float tile[BLK][DIM + 1];
  const uint64_t b = blockIdx.x;
  for (int i = threadIdx.x; i < BLK * DIM; i += blockDim.x) {
    int r = i / DIM, d = i % DIM;
    uint64_t p = b * BLK + r;
    tile[r][d] = p < n ? vecs[(uint64_t)perm[p] * DIM + d] : 0.f;
  }
  __syncthreads();
  float *out = blocks + b * BLK_FLOATS;
  for (int i = threadIdx.x; i < BLK * DIM; i += blockDim.x) {
    int d = i / BLK, r = i % BLK;
    out[d * BLK + r] = tile[r][d];
  }
  for (int r = threadIdx.x; r < BLK; r += blockDim.x) {
    uint64_t p = b * BLK + r;
    out[DIM * BLK + r] = p < n ? norms[perm[p]] : 0.f;
  }
}

// distinct labels: starts of the label runs of the category order
__global__ void k_label_runs(const int32_t *__restrict__ lab, uint64_t n, uint32_t *__restrict__ count) {
  uint32_t c = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    c += (i == 0 || lab[i] != lab[i - 1]) ? 1u : 0u;
  if (c) atomicAdd(count, c);
}

inline unsigned grid_for(uint64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

int radix_sort_pairs(fknn_index *idx, uint32_t *keys, uint32_t *vals, uint32_t *keys_tmp, uint32_t *vals_tmp,
                     uint64_t n, int begin_bit, int end_bit, cudaStream_t st) {
  if (n == 0) return FKNN_OK;
  const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
  uint32_t *hist = nullptr;
  int rc = ws_get(idx, 15, (size_t)ntiles * RS_DIGITS * sizeof(uint32_t), (void **)&hist);
  if (rc) return rc;
  uint32_t *ki = keys, *vi = vals, *ko = keys_tmp, *vo = vals_tmp;
  for (int shift = begin_bit; shift < end_bit; shift += RS_BITS) {
    rs_hist<<<ntiles, RS_THREADS, 0, st>>>(ki, n, shift, hist, ntiles);
    rs_scan<<<1, 1024, 0, st>>>(hist, (uint64_t)ntiles * RS_DIGITS);
    rs_scatter<<<ntiles, RS_THREADS, 0, st>>>(ki, vi, ko, vo, n, shift, hist, ntiles);
    g_launches += 3;
    uint32_t *t;
    t = ki; ki = ko; ko = t;
    t = vi; vi = vo; vo = t;
  }
  if (ki != keys) {
    FKNN_CUDA(cudaMemcpyAsync(keys, ki, n * 4, cudaMemcpyDeviceToDevice, st));
    FKNN_CUDA(cudaMemcpyAsync(vals, vi, n * 4, cudaMemcpyDeviceToDevice, st));
  }
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

int alloc_index_columns(fknn_index *idx) {
  const uint64_t n = idx->n;
  int rc;
  if ((rc = dev_alloc(idx, (void **)&idx->vecs, n * DIM * sizeof(float)))) return rc;
  if ((rc = dev_alloc(idx, (void **)&idx->norms, n * sizeof(float)))) return rc;
  if ((rc = dev_alloc(idx, (void **)&idx->labels_f, n * sizeof(float)))) return rc;
  if ((rc = dev_alloc(idx, (void **)&idx->ts_f, n * sizeof(float)))) return rc;
  return FKNN_OK;
}

int build_index(fknn_index *idx, const float *h_vecs, const float *h_labels, const float *h_ts, cudaStream_t st) {
  const uint64_t n = idx->n;
  int rc;
  if ((rc = alloc_index_columns(idx))) return rc;
  FKNN_CUDA(cudaMemcpyAsync(idx->vecs, h_vecs, n * DIM * sizeof(float), cudaMemcpyDefault, st));
  FKNN_CUDA(cudaMemcpyAsync(idx->labels_f, h_labels, n * sizeof(float), cudaMemcpyDefault, st));
  FKNN_CUDA(cudaMemcpyAsync(idx->ts_f, h_ts, n * sizeof(float), cudaMemcpyDefault, st));
  return build_index_from_columns(idx, st);
}

int build_index_from_columns(fknn_index *idx, cudaStream_t st) {
  const uint64_t n = idx->n;
  int rc;
  FKNN_CUDA(cudaMemsetAsync(idx->d_flag, 0, sizeof(int), st));
  k_validate_base<<<148 * 8, 256, 0, st>>>(idx->vecs, idx->labels_f, idx->ts_f, n, idx->d_flag);
  int flag = 0;
  FKNN_CUDA(cudaMemcpyAsync(&flag, idx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  if (flag) {
    set_error(std::string("fknn_index_create: ") + ((flag & 1) ? "vector value not finite or above 1e15; " : "") +
              ((flag & 2) ? "label not finite or outside int32; " : "") + ((flag & 4) ? "timestamp not finite" : ""));
    return FKNN_EINVAL;
  }
  k_norms<<<grid_for(n, 256), 256, 0, st>>>(idx->vecs, n, idx->norms);

  uint32_t *keys, *vals, *ktmp, *vtmp;
  if ((rc = ws_get(idx, 11, n * 4, (void **)&keys))) return rc;
  if ((rc = ws_get(idx, 12, n * 4, (void **)&vals))) return rc;
  if ((rc = ws_get(idx, 13, n * 4, (void **)&ktmp))) return rc;
  if ((rc = ws_get(idx, 14, n * 4, (void **)&vtmp))) return rc;

  idx->nblk = (uint32_t)((n + BLK - 1) / BLK);
  for (int o = 0; o < 2; ++o) {
    OrderData &od = idx->ord[o];
    if ((rc = dev_alloc(idx, (void **)&od.perm, n * 4))) return rc;
    if ((rc = dev_alloc(idx, (void **)&od.ts, n * 4))) return rc;
    if ((rc = dev_alloc(idx, (void **)&od.label, n * 4))) return rc;
    if ((rc = dev_alloc(idx, (void **)&od.blocks, (size_t)idx->nblk * BLK_BYTES))) return rc;
  }
  // time order: stable sort of (ts, id) keys starting from the identity
  k_time_keys<<<grid_for(n, 256), 256, 0, st>>>(idx->ts_f, n, keys, vals);
  g_launches += 3;
  if ((rc = radix_sort_pairs(idx, keys, vals, ktmp, vtmp, n, 0, 32, st))) return rc;
  FKNN_CUDA(cudaMemcpyAsync(idx->ord[ORDER_TIME].perm, vals, n * 4, cudaMemcpyDeviceToDevice, st));
  // category order: stable sort by label of the time order -> (label, ts, id)
  k_label_keys<<<grid_for(n, 256), 256, 0, st>>>(idx->labels_f, idx->ord[ORDER_TIME].perm, n, keys, vals);
  g_launches += 1;
  if ((rc = radix_sort_pairs(idx, keys, vals, ktmp, vtmp, n, 0, 32, st))) return rc;
  FKNN_CUDA(cudaMemcpyAsync(idx->ord[ORDER_CAT].perm, vals, n * 4, cudaMemcpyDeviceToDevice, st));

  for (int o = 0; o < 2; ++o) {
    OrderData &od = idx->ord[o];
    k_order_columns<<<grid_for(n, 256), 256, 0, st>>>(od.perm, idx->ts_f, idx->labels_f, n, od.ts, od.label);
    k_build_blocks<<<idx->nblk, 256, 0, st>>>(idx->vecs, idx->norms, od.perm, n, od.blocks);
    g_launches += 2;
  }
  FKNN_CUDA(cudaMemsetAsync(idx->d_flag, 0, sizeof(int), st));
  k_label_runs<<<148 * 4, 256, 0, st>>>(idx->ord[ORDER_CAT].label, n, reinterpret_cast<uint32_t *>(idx->d_flag));
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  uint32_t runs = 0;
  FKNN_CUDA(cudaMemcpyAsync(&runs, idx->d_flag, 4, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaMemsetAsync(idx->d_flag, 0, sizeof(int), st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  idx->n_labels = runs ? runs : 1;
  return FKNN_OK;
}

}  // namespace fknn
