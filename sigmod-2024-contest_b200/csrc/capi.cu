// C ABI entry points (include/fknn.h), error plumbing and device memory.
#include <cstdio>
#include <cstring>
#include <functional>
#include <new>

#include "fknn_internal.cuh"

namespace fknn {

thread_local uint32_t g_launches = 0;
static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }

int cuda_fail(cudaError_t e, const char *what) {
  g_err = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") in " + what;
  if (e == cudaErrorMemoryAllocation) return FKNN_ENOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return FKNN_ENODEV;
  return FKNN_ECUDA;
}

int dev_alloc(fknn_index *idx, void **p, size_t bytes) {
  if (idx->hbm_budget && idx->bytes + bytes > idx->hbm_budget) {
    set_error("device allocation of " + std::to_string(bytes) + " bytes exceeds the index HBM budget of " +
              std::to_string(idx->hbm_budget));
    return FKNN_ENOMEM;
  }
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_fail(e, "cudaMalloc");
  }
  idx->bytes += bytes;
  return FKNN_OK;
}

static void dev_free(fknn_index *idx, void *p, size_t bytes) {
  if (p) {
    cudaFree(p);
    idx->bytes -= bytes;
  }
}

int ws_get(fknn_index *idx, int slot, size_t bytes, void **p) {
  DevBuf &b = idx->ws[slot];
  if (b.bytes < bytes) {
    // in-flight work may still read the old buffer
    cudaDeviceSynchronize();
    dev_free(idx, b.p, b.bytes);
    b.p = nullptr;
    b.bytes = 0;
    size_t want = bytes + bytes / 4;
    int rc = dev_alloc(idx, &b.p, want);
    if (rc) return rc;
    b.bytes = want;
  }
  *p = b.p;
  return FKNN_OK;
}

int hs_get(fknn_index *idx, int slot, size_t bytes, void **p) {
  HostBuf &b = idx->hs[slot];
  if (b.bytes < bytes) {
    cudaDeviceSynchronize();
    if (b.p) cudaFreeHost(b.p);
    b.p = nullptr;
    b.bytes = 0;
    size_t want = bytes + bytes / 4 + 64;
    cudaError_t e = cudaMallocHost(&b.p, want);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
    b.bytes = want;
  }
  *p = b.p;
  return FKNN_OK;
}

MemLoc mem_loc(const void *p, int dev) {
  if (!p) return MemLoc::Host;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return MemLoc::Host;
  }
  if (a.type == cudaMemoryTypeManaged) return MemLoc::Here;
  if (a.type == cudaMemoryTypeDevice) return a.device == dev ? MemLoc::Here : MemLoc::Other;
  return MemLoc::Host;
}

int check_local_buffers(const char *fn, int dev, std::initializer_list<const void *> bufs) {
  for (const void *p : bufs)
    if (p && mem_loc(p, dev) == MemLoc::Other) {
      set_error(std::string(fn) + ": a buffer is device memory of another device (device " + std::to_string(dev) +
                " runs this call)");
      return FKNN_EINVAL;
    }
  return FKNN_OK;
}

static bool is_device_ptr(const void *p, int dev) { return mem_loc(p, dev) == MemLoc::Here; }

static void free_index(fknn_index *idx) {
  if (!idx) return;
  cudaSetDevice(idx->device);
  cudaDeviceSynchronize();
  idx->graph.release();
  if (idx->graph.cap) cudaStreamDestroy(idx->graph.cap);
  if (idx->graph.side) cudaStreamDestroy(idx->graph.side);
  if (idx->graph.fork) cudaEventDestroy(idx->graph.fork);
  if (idx->graph.join) cudaEventDestroy(idx->graph.join);
  if (idx->side_stream) cudaStreamDestroy(idx->side_stream);
  if (idx->ev_fork) cudaEventDestroy(idx->ev_fork);
  if (idx->ev_join) cudaEventDestroy(idx->ev_join);
  if (idx->is_view) {
    for (auto &b : idx->ws) cudaFree(b.p);
    for (auto &b : idx->hs)
      if (b.p) cudaFreeHost(b.p);
    cudaFree(idx->d_flag);
    delete idx;
    return;
  }
  cudaFree(idx->vecs);
  cudaFree(idx->norms);
  cudaFree(idx->labels_f);
  cudaFree(idx->ts_f);
  for (int o = 0; o < 2; ++o) {
    cudaFree(idx->ord[o].blocks);
    cudaFree(idx->ord[o].perm);
    cudaFree(idx->ord[o].ts);
    cudaFree(idx->ord[o].label);
    cudaFree(idx->bf16_blocks[o]);
    cudaFree(idx->fp8_blocks[o]);
  }
  cudaFree(idx->fp8_scale);
  for (auto &b : idx->ws) cudaFree(b.p);
  for (auto &b : idx->hs)
    if (b.p) cudaFreeHost(b.p);
  cudaFree(idx->d_flag);
  if (idx->own_stream) cudaStreamDestroy(idx->own_stream);
  delete idx;
}

int make_index_view(fknn_index *base, fknn_index **out) {
  *out = nullptr;
  fknn_index *v = new (std::nothrow) fknn_index();
  if (!v) {
    set_error("out of host memory");
    return FKNN_ENOMEM;
  }
  v->device = base->device;
  v->n = base->n;
  v->nblk = base->nblk;
  v->vecs = base->vecs;
  v->norms = base->norms;
  v->labels_f = base->labels_f;
  v->ts_f = base->ts_f;
  for (int o = 0; o < 2; ++o) {
    v->ord[o] = base->ord[o];
    v->bf16_blocks[o] = base->bf16_blocks[o];
    v->fp8_blocks[o] = base->fp8_blocks[o];
  }
  v->fp8_scale = base->fp8_scale;
  for (int m = 0; m < 3; ++m) v->tuning[m] = base->tuning[m];
  v->num_sms = base->num_sms;
  v->n_labels = base->n_labels;
  v->is_view = true;
  cudaError_t e = cudaSetDevice(v->device);
  if (e == cudaSuccess) e = cudaMalloc(&v->d_flag, 64);
  if (e != cudaSuccess) {
    delete v;
    return cuda_fail(e, "cudaMalloc");
  }
  *out = v;
  return FKNN_OK;
}

void destroy_index(fknn_index *idx) { free_index(idx); }

void trim_scratch(fknn_index *idx) {
  std::lock_guard<std::mutex> lock(idx->mu);
  cudaSetDevice(idx->device);
  for (auto &w : idx->ws) {
    dev_free(idx, w.p, w.bytes);
    w.p = nullptr;
    w.bytes = 0;
  }
}

uint64_t scratch_bytes(const fknn_index *idx) {
  uint64_t b = 0;
  for (const auto &w : idx->ws) b += w.bytes;
  return b;
}

// Device set-up, the row columns and orders (build), the reduced-precision
// copies the options ask for, then the build temporaries are released.
int create_index(uint64_t n, const fknn_index_opts *opts,
                 const std::function<int(fknn_index *, cudaStream_t)> &build, fknn_index **out) {
  if (n == 0 || n >= (1ull << 31)) {
    set_error("fknn_index_create: n must be in [1, 2^31)");
    return FKNN_EINVAL;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("fknn_index_create: no CUDA device");
    return FKNN_ENODEV;
  }
  fknn_index *idx = new (std::nothrow) fknn_index();
  if (!idx) return FKNN_ENOMEM;
  idx->device = opts ? opts->device : 0;
  idx->hbm_budget = opts ? opts->hbm_budget : 0;
  idx->n = n;
  if (idx->device < 0 || idx->device >= ndev) {
    delete idx;
    set_error("fknn_index_create: bad device ordinal");
    return FKNN_EINVAL;
  }
  int rc = FKNN_OK;
  e = cudaSetDevice(idx->device);
  if (e != cudaSuccess) rc = cuda_fail(e, "cudaSetDevice");
  if (!rc) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, idx->device) == cudaSuccess && sms > 0)
      idx->num_sms = sms;
    e = cudaStreamCreateWithFlags(&idx->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamCreate");
  }
  if (!rc) {
    e = cudaMalloc(&idx->d_flag, 64);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc");
  }
  if (!rc) rc = build(idx, idx->own_stream);
  if (!rc && opts && opts->build_bf16) {
    rc = build_bf16(idx, idx->own_stream);
    if (!rc) {
      cudaError_t e2 = cudaStreamSynchronize(idx->own_stream);
      if (e2 != cudaSuccess) rc = cuda_fail(e2, "build_bf16");
    }
  }
  if (!rc && opts && opts->build_fp8) {
    rc = build_fp8(idx, idx->own_stream);
    if (!rc) {
      cudaError_t e2 = cudaStreamSynchronize(idx->own_stream);
      if (e2 != cudaSuccess) rc = cuda_fail(e2, "build_fp8");
    }
  }
  // build temporaries are not needed by searches
  for (int s = 10; s < 16; ++s) {
    if (idx->ws[s].p) {
      cudaFree(idx->ws[s].p);
      idx->bytes -= idx->ws[s].bytes;
      idx->ws[s].p = nullptr;
      idx->ws[s].bytes = 0;
    }
  }
  if (rc) {
    free_index(idx);
    return rc;
  }
  *out = idx;
  return FKNN_OK;
}

}  // namespace fknn

using namespace fknn;

extern "C" {

int fknn_version(void) { return 100; }

const char *fknn_last_error(void) { return g_err.c_str(); }

int fknn_index_create(const float *vecs, const float *labels, const float *ts, uint64_t n, uint32_t dim,
                      const fknn_index_opts *opts, fknn_index **out) {
  g_err.clear();
  g_launches = 0;
  if (!out) {
    set_error("fknn_index_create: out is NULL");
    return FKNN_EINVAL;
  }
  *out = nullptr;
  if (dim != (uint32_t)DIM) {
    set_error("fknn_index_create: dim must be 100");
    return FKNN_EINVAL;
  }
  if (!vecs || !labels || !ts) {
    set_error("fknn_index_create: NULL input column");
    return FKNN_EINVAL;
  }
  return create_index(n, opts, [&](fknn_index *idx, cudaStream_t st) { return build_index(idx, vecs, labels, ts, st); },
                      out);
}

int fknn_index_destroy(fknn_index *index) {
  free_index(index);
  return FKNN_OK;
}

int fknn_index_bytes(const fknn_index *index, uint64_t *bytes) {
  if (!index || !bytes) return FKNN_EINVAL;
  *bytes = index->bytes;
  return FKNN_OK;
}

int fknn_search_ex(fknn_index *idx, const float *qvecs, const float *metas, uint32_t nq, uint32_t k,
                   const fknn_search_opts *opts, uint32_t *ids, float *dists, void *stream, fknn_search_stats *stats) {
  g_err.clear();
  g_launches = 0;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (!idx) {
    set_error("fknn_search: NULL index");
    return FKNN_EINVAL;
  }
  const int mode = opts ? opts->mode : FKNN_MODE_EXACT_FP32;
  if (k == 0 || k > (uint32_t)KMAX_TILE) {
    set_error("fknn_search: k must be in [1, 128]");
    return FKNN_EINVAL;
  }
  if (nq == 0) return FKNN_OK;
  if (!qvecs || !metas || !ids) {
    set_error("fknn_search: NULL qvecs/metas/ids");
    return FKNN_EINVAL;
  }
  const uint32_t kprime = (opts && opts->kprime) ? opts->kprime : 400;
  if (opts && (opts->flags & ~FKNN_SEARCH_GRAPH)) {
    set_error("fknn_search: unknown flag in fknn_search_opts.flags");
    return FKNN_EINVAL;
  }
  if (mode == FKNN_MODE_BF16_RERANK || mode == FKNN_MODE_FP8_RERANK) {
    if (mode == FKNN_MODE_BF16_RERANK ? !idx->bf16_blocks[0] : !idx->fp8_blocks[0]) {
      set_error(mode == FKNN_MODE_BF16_RERANK ? "fknn_search: BF16 mode needs an index created with build_bf16"
                                             : "fknn_search: FP8 mode needs an index created with build_fp8");
      return FKNN_EUNSUPPORTED;
    }
    if (kprime < k || kprime > 1024) {
      set_error("fknn_search: kprime must be in [k, 1024]");
      return FKNN_EINVAL;
    }
  } else if (mode != FKNN_MODE_EXACT_FP32) {
    set_error("fknn_search: mode not built into this index");
    return FKNN_EUNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(idx->mu);
  FKNN_CUDA(cudaSetDevice(idx->device));
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  const float *d_q = qvecs, *d_meta = metas;
  uint32_t *d_ids = ids;
  float *d_dists = dists;
  const int dev = idx->device;
  if ((rc = check_local_buffers("fknn_search", dev, {qvecs, metas, ids, dists}))) return rc;
  const bool q_dev = is_device_ptr(qvecs, dev), m_dev = is_device_ptr(metas, dev);
  const bool i_dev = is_device_ptr(ids, dev), dd_dev = dists ? is_device_ptr(dists, dev) : true;
  if (!q_dev) {
    if ((rc = ws_get(idx, 0, (size_t)nq * DIM * 4, (void **)&d_q))) return rc;
    FKNN_CUDA(cudaMemcpyAsync((void *)d_q, qvecs, (size_t)nq * DIM * 4, cudaMemcpyHostToDevice, st));
  }
  if (!m_dev) {
    if ((rc = ws_get(idx, 1, (size_t)nq * 16, (void **)&d_meta))) return rc;
    FKNN_CUDA(cudaMemcpyAsync((void *)d_meta, metas, (size_t)nq * 16, cudaMemcpyHostToDevice, st));
  }
  if (!i_dev)
    if ((rc = ws_get(idx, 8, (size_t)nq * k * 4, (void **)&d_ids))) return rc;
  if (dists && !dd_dev)
    if ((rc = ws_get(idx, 9, (size_t)nq * k * 4, (void **)&d_dists))) return rc;
  const bool graph = opts && (opts->flags & FKNN_SEARCH_GRAPH);
  if (mode == FKNN_MODE_BF16_RERANK)
    rc = (graph ? search_bf16_graph : search_bf16)(idx, d_q, d_meta, nq, k, kprime, d_ids, d_dists, st, stats);
  else if (mode == FKNN_MODE_FP8_RERANK)
    rc = (graph ? search_fp8_graph : search_fp8)(idx, d_q, d_meta, nq, k, kprime, d_ids, d_dists, st, stats);
  else
    rc = search_exact(idx, d_q, d_meta, nq, k, d_ids, d_dists, st, stats);
  // on a failure the short-slab scans may still be writing the outputs
  if (rc && idx->side_stream) cudaStreamSynchronize(idx->side_stream);
  if (rc) return rc;
  if (!i_dev) FKNN_CUDA(cudaMemcpyAsync(ids, d_ids, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, st));
  if (dists && !dd_dev) FKNN_CUDA(cudaMemcpyAsync(dists, d_dists, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, st));
  int flag = 0;
  FKNN_CUDA(cudaMemcpyAsync(&flag, idx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  if (stats) stats->kernel_launches = g_launches;
  if (flag & (1 << 8)) {
    // the outputs are complete: the affected queries were re-answered by the
    // exact scan; the status tells the caller that a device wait gave up
    set_error("fknn_search: a bounded device wait gave up; affected queries were answered by the exact scan");
    return FKNN_ETIMEOUT;
  }
  return FKNN_OK;
}

int fknn_index_test_withhold_copy(fknn_index *index) {
  if (!index) return FKNN_EINVAL;
  std::lock_guard<std::mutex> lock(index->mu);
  index->test_withhold = true;
  return FKNN_OK;
}

int fknn_index_set_tuning(fknn_index *index, int mode, const fknn_tuning *t) {
  if (!index || !t || mode < 0 || mode > 2) {
    set_error("fknn_index_set_tuning: NULL argument or unknown mode");
    return FKNN_EINVAL;
  }
  if ((t->list_slack && (t->list_slack < 256 || t->list_slack > 1024)) || t->items_per_sm > 64 ||
      t->min_chunk_blocks > 4096 || t->bound_refresh > 4096 || t->pilot_stride > 1024) {
    set_error("fknn_index_set_tuning: list_slack in [256, 1024], items_per_sm <= 64, min_chunk_blocks <= 4096, "
              "bound_refresh <= 4096, pilot_stride <= 1024");
    return FKNN_EINVAL;
  }
  std::lock_guard<std::mutex> lock(index->mu);
  fknn_tuning &d = index->tuning[mode];
  if (t->list_slack) d.list_slack = t->list_slack;
  if (t->items_per_sm) d.items_per_sm = t->items_per_sm;
  if (t->min_chunk_blocks) d.min_chunk_blocks = t->min_chunk_blocks;
  d.bound_refresh = t->bound_refresh;
  d.pilot_stride = t->pilot_stride;
  return FKNN_OK;
}

int fknn_index_get_tuning(const fknn_index *index, int mode, fknn_tuning *t) {
  if (!index || !t || mode < 0 || mode > 2) {
    set_error("fknn_index_get_tuning: NULL argument or unknown mode");
    return FKNN_EINVAL;
  }
  *t = index->tuning[mode];
  return FKNN_OK;
}

int fknn_search(fknn_index *index, const float *qvecs, const float *metas, uint32_t nq, uint32_t k, int mode,
                uint32_t *ids, float *dists, void *stream) {
  fknn_search_opts o{};
  o.mode = mode;
  o.kprime = 0;
  return fknn_search_ex(index, qvecs, metas, nq, k, &o, ids, dists, stream, nullptr);
}

int fknn_count_matches(fknn_index *idx, const float *metas, uint32_t nq, uint32_t *counts, void *stream) {
  g_err.clear();
  g_launches = 0;
  if (!idx || !metas || !counts) return FKNN_EINVAL;
  if (nq == 0) return FKNN_OK;
  std::lock_guard<std::mutex> lock(idx->mu);
  FKNN_CUDA(cudaSetDevice(idx->device));
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  const float *d_meta = metas;
  uint32_t *d_c = counts;
  if ((rc = check_local_buffers("fknn_count_matches", idx->device, {metas, counts}))) return rc;
  const bool m_dev = is_device_ptr(metas, idx->device), c_dev = is_device_ptr(counts, idx->device);
  if (!m_dev) {
    if ((rc = ws_get(idx, 1, (size_t)nq * 16, (void **)&d_meta))) return rc;
    FKNN_CUDA(cudaMemcpyAsync((void *)d_meta, metas, (size_t)nq * 16, cudaMemcpyHostToDevice, st));
  }
  if (!c_dev)
    if ((rc = ws_get(idx, 8, (size_t)nq * 4, (void **)&d_c))) return rc;
  // reuse the query validator with a zero vector block is not needed: only metas
  if ((rc = count_matches(idx, d_meta, nq, d_c, st))) return rc;
  if (!c_dev) FKNN_CUDA(cudaMemcpyAsync(counts, d_c, (size_t)nq * 4, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  return FKNN_OK;
}

int fknn_filter_rows(fknn_index *idx, const float *meta4, uint32_t *out_ids, uint64_t *count, void *stream) {
  g_err.clear();
  g_launches = 0;
  if (!idx || !meta4 || !out_ids || !count) return FKNN_EINVAL;
  int rc;
  if ((rc = filter_check_preds(meta4, 1, "fknn_filter_rows"))) return rc;
  std::lock_guard<std::mutex> lock(idx->mu);
  FKNN_CUDA(cudaSetDevice(idx->device));
  cudaStream_t st = (cudaStream_t)stream;
  uint32_t *d_out = out_ids;
  if ((rc = check_local_buffers("fknn_filter_rows", idx->device, {out_ids}))) return rc;
  const bool o_dev = is_device_ptr(out_ids, idx->device);
  if (!o_dev)
    if ((rc = ws_get(idx, 8, (size_t)idx->n * 4, (void **)&d_out))) return rc;
  if ((rc = filter_rows(idx, meta4, d_out, count, st))) return rc;
  if (!o_dev && *count) FKNN_CUDA(cudaMemcpyAsync(out_ids, d_out, *count * 4, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  return FKNN_OK;
}

int fknn_filter_rows_batch(fknn_index *idx, const float *metas, uint32_t np, uint32_t *out_ids, uint64_t *counts,
                           void *stream) {
  g_err.clear();
  g_launches = 0;
  if (!idx || !metas || !out_ids || !counts) {
    set_error("fknn_filter_rows_batch: NULL argument");
    return FKNN_EINVAL;
  }
  int rc;
  if ((rc = filter_check_preds(metas, np, "fknn_filter_rows_batch"))) return rc;
  if (np == 0) return FKNN_OK;
  std::lock_guard<std::mutex> lock(idx->mu);
  FKNN_CUDA(cudaSetDevice(idx->device));
  if (!is_device_ptr(out_ids, idx->device) || !is_device_ptr(counts, idx->device)) {
    set_error("fknn_filter_rows_batch: out_ids and counts must be device memory of the index's device");
    return FKNN_EINVAL;
  }
  return filter_rows_batch(idx, metas, np, out_ids, counts, (cudaStream_t)stream);
}

int fknn_bruteforce_rows(const float *nodes, uint32_t n, const float *queries, uint32_t nq, uint32_t *gt) {
  g_err.clear();
  if (!nodes || !queries || !gt || n == 0) {
    set_error("fknn_bruteforce_rows: bad arguments");
    return FKNN_EINVAL;
  }
  // split the contest rows into the columns the index takes
  std::vector<float> vecs((size_t)n * DIM), labels(n), ts(n), qv((size_t)nq * DIM), meta((size_t)nq * 4);
  for (uint32_t i = 0; i < n; ++i) {
    const float *r = nodes + (size_t)i * (DIM + 2);
    labels[i] = r[0];
    ts[i] = r[1];
    std::memcpy(&vecs[(size_t)i * DIM], r + 2, DIM * 4);
  }
  for (uint32_t i = 0; i < nq; ++i) {
    const float *r = queries + (size_t)i * (DIM + 4);
    std::memcpy(&meta[(size_t)i * 4], r, 16);
    std::memcpy(&qv[(size_t)i * DIM], r + 4, DIM * 4);
  }
  fknn_index *idx = nullptr;
  fknn_index_opts o;
  std::memset(&o, 0, sizeof(o));
  int rc = fknn_index_create(vecs.data(), labels.data(), ts.data(), n, DIM, &o, &idx);
  if (rc) return rc;
  rc = fknn_search(idx, qv.data(), meta.data(), nq, 100, FKNN_MODE_EXACT_FP32, gt, nullptr, nullptr);
  std::string keep = g_err;
  fknn_index_destroy(idx);
  g_err = keep;
  return rc;
}

}  // extern "C"
