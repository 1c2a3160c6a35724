// FP32 re-rank of candidate lists: the step that follows every approximate
// search in the reference (hybrid_graph.cpp:216-228, 284-296, 481-492: the
// graph's or the SQ8 scan's candidates re-scored in FP32 and the k best
// kept).  One block per query: exact distances with the reference's
// normal_l2 arithmetic (distance.h:62-72), duplicates dropped, the k
// smallest by (distance, id) written ascending.
#include "device_util.cuh"

namespace fknn {
namespace {

constexpr int RK_THREADS = 256;
constexpr int RK_MAXC = 2048;  // candidates per query

__global__ void __launch_bounds__(RK_THREADS)
    k_rerank(const float *__restrict__ vecs, uint64_t n, const float *__restrict__ q, uint32_t nq,
             const uint32_t *__restrict__ cand, uint32_t nc, uint32_t k, uint32_t *__restrict__ ids,
             float *__restrict__ dists, int *err) {
  __shared__ uint64_t key[RK_MAXC];
  __shared__ float qv[DIM];
  __shared__ uint32_t keep[RK_THREADS + 1];
  const int tid = threadIdx.x;
  const uint32_t qi = blockIdx.x;
  for (int d = tid; d < DIM; d += RK_THREADS) qv[d] = q[(uint64_t)qi * DIM + d];
  int np2 = 32;
  while (np2 < (int)nc) np2 <<= 1;
  __syncthreads();
  for (int i = tid; i < np2; i += RK_THREADS) {
    uint64_t kk = ~0ull;
    if (i < (int)nc) {
      const uint32_t id = cand[(uint64_t)qi * nc + i];
      if (id < n) kk = exact_key(seq_l2_strided(vecs + (uint64_t)id * DIM, 1, qv), id);
      else if (id != 0xffffffffu) atomicOr(err, ERR_BAD_QUERY_VALUE);
    }
    key[i] = kk;
  }
  __syncthreads();
  block_bitonic_sort(key, np2);
  // drop repeated ids (equal keys are adjacent), keep order, first k
  const int per = (np2 + RK_THREADS - 1) / RK_THREADS;
  const int i0 = tid * per, i1 = min(i0 + per, np2);
  uint32_t c = 0;
  for (int i = i0; i < i1; ++i) c += key[i] != ~0ull && (i == 0 || key[i] != key[i - 1]);
  keep[tid + 1] = c;
  if (tid == 0) keep[0] = 0;
  __syncthreads();
  if (tid == 0)
    for (int t = 0; t < RK_THREADS; ++t) keep[t + 1] += keep[t];
  __syncthreads();
  uint32_t w = keep[tid];
  for (int i = i0; i < i1 && w < k; ++i)
    if (key[i] != ~0ull && (i == 0 || key[i] != key[i - 1])) {
      ids[(uint64_t)qi * k + w] = (uint32_t)key[i];
      if (dists) dists[(uint64_t)qi * k + w] = sortable_f32((uint32_t)(key[i] >> 32));
      ++w;
    }
  for (uint32_t j = keep[RK_THREADS] + tid; j < k; j += RK_THREADS) {
    ids[(uint64_t)qi * k + j] = 0xffffffffu;
    if (dists) dists[(uint64_t)qi * k + j] = INFINITY;
  }
}

bool dev_ptr(const void *p, int dev) { return mem_loc(p, dev) == MemLoc::Here; }

}  // namespace

int launch_rerank(fknn_index *idx, const float *d_q, uint32_t nq, const uint32_t *d_cand, uint32_t nc, uint32_t k,
                  uint32_t *d_ids, float *d_dists, int *d_err, cudaStream_t st) {
  if (nq == 0) return FKNN_OK;
  if (nc == 0 || nc > (uint32_t)RK_MAXC || k == 0 || k > nc) {
    set_error("re-rank: need 1 <= k <= nc <= 2048");
    return FKNN_EINVAL;
  }
  k_rerank<<<nq, RK_THREADS, 0, st>>>(idx->vecs, idx->n, d_q, nq, d_cand, nc, k, d_ids, d_dists, d_err);
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  return FKNN_OK;
}

}  // namespace fknn

using namespace fknn;

extern "C" int fknn_rerank(fknn_index *idx, const float *qvecs, uint32_t nq, const uint32_t *cand, uint32_t nc,
                           uint32_t k, uint32_t *ids, float *dists, void *stream) {
  g_launches = 0;
  if (!idx || !qvecs || !cand || !ids) {
    set_error("fknn_rerank: NULL argument");
    return FKNN_EINVAL;
  }
  if (nc == 0 || nc > (uint32_t)RK_MAXC || k == 0 || k > nc) {
    set_error("fknn_rerank: need 1 <= k <= nc <= 2048");
    return FKNN_EINVAL;
  }
  if (nq == 0) return FKNN_OK;
  std::lock_guard<std::mutex> lock(idx->mu);
  FKNN_CUDA(cudaSetDevice(idx->device));
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  const float *d_q = qvecs;
  const uint32_t *d_c = cand;
  uint32_t *d_ids = ids;
  float *d_d = dists;
  const int dev = idx->device;
  if ((rc = check_local_buffers("fknn_rerank", dev, {qvecs, cand, ids, dists}))) return rc;
  const bool q_dev = dev_ptr(qvecs, dev), c_dev = dev_ptr(cand, dev), i_dev = dev_ptr(ids, dev);
  const bool dd_dev = dists ? dev_ptr(dists, dev) : true;
  if (!q_dev) {
    if ((rc = ws_get(idx, 0, (size_t)nq * DIM * 4, (void **)&d_q))) return rc;
    FKNN_CUDA(cudaMemcpyAsync((void *)d_q, qvecs, (size_t)nq * DIM * 4, cudaMemcpyHostToDevice, st));
  }
  if (!c_dev) {
    if ((rc = ws_get(idx, 1, (size_t)nq * nc * 4, (void **)&d_c))) return rc;
    FKNN_CUDA(cudaMemcpyAsync((void *)d_c, cand, (size_t)nq * nc * 4, cudaMemcpyHostToDevice, st));
  }
  if (!i_dev)
    if ((rc = ws_get(idx, 8, (size_t)nq * k * 4, (void **)&d_ids))) return rc;
  if (dists && !dd_dev)
    if ((rc = ws_get(idx, 9, (size_t)nq * k * 4, (void **)&d_d))) return rc;
  FKNN_CUDA(cudaMemsetAsync(idx->d_flag, 0, 4, st));
  k_rerank<<<nq, RK_THREADS, 0, st>>>(idx->vecs, idx->n, d_q, nq, d_c, nc, k, d_ids, d_d, idx->d_flag);
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  if (!i_dev) FKNN_CUDA(cudaMemcpyAsync(ids, d_ids, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, st));
  if (dists && !dd_dev) FKNN_CUDA(cudaMemcpyAsync(dists, d_d, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, st));
  int flag = 0;
  FKNN_CUDA(cudaMemcpyAsync(&flag, idx->d_flag, 4, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  if (flag) {
    set_error("fknn_rerank: a candidate id is neither a row of the index nor UINT32_MAX");
    return FKNN_EINVAL;
  }
  return FKNN_OK;
}
