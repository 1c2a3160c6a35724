// Symmetric SQ8 (pyglass/glass/quant/sq8_sym_quant.hpp) and the SQ8 slab
// brute force (bruteforce.h:244-289) on the GPU.
//
// bruteforce() returns the reference's maxPQIFCS heap array, which depends
// on the exact insertion history (ties on the int distance are frequent).
// The kernel reproduces it: one block per query scans the slab in chunks of
// 1024 codes; every code whose distance is below the heap root at the start
// of its chunk (the only ones must_pop_emplace can admit, since the root
// only falls) is compacted in slab order with warp ballots and replayed on a
// shared-memory copy of the heap by one thread, with the reference's
// emplace / push_down steps.  The distance itself is an exact int32
// sum over 112 bytes from dp4a: |q-c|^2 = |q|^2 + |c|^2 - 2 q.c.
#include "device_util.cuh"

namespace fknn {

namespace {

constexpr int SQ8_CODE = 112;
constexpr int SQ8_WORDS = SQ8_CODE / 4;
constexpr int BF_THREADS = 256;
constexpr int BF_CHUNK = 1024;
constexpr int BF_KMAX = 2048;

__global__ void k_absmax(const float *__restrict__ x, uint64_t count, uint32_t *__restrict__ out) {
  float m = 0.f;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(x[i]));
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));  // non-negative floats order as uints
}

// sq8_sym_quant.hpp:63-74: x / alpha (IEEE division), clamp to [-1, 1],
// std::round(x * 127) (half away from zero), dims 100..111 zero.
__global__ void k_sq8_encode(const float *__restrict__ x, uint64_t n, float alpha, int8_t *__restrict__ codes) {
  const uint64_t total = n * SQ8_CODE;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i / SQ8_CODE;
    const int d = (int)(i % SQ8_CODE);
    int8_t c = 0;
    if (d < DIM) {
      float y = __fdiv_rn(x[r * DIM + d], alpha);
      if (y > 1.0f) y = 1.0f;
      if (y < -1.0f) y = -1.0f;
      c = (int8_t)roundf(__fmul_rn(y, 127.0f));
    }
    codes[i] = c;
  }
}

struct HeapNode {
  int d;
  int id;
};

// maxPQIFCS::push_down (bruteforce.h:78-87) on a 1-based array.
__device__ __forceinline__ void heap_push_down(HeapNode *h, int cnt, int x) {
  while ((x << 1) <= cnt) {
    int t = x << 1;
    if ((t | 1) <= cnt && h[t | 1].d > h[t].d) t |= 1;
    if (h[t].d <= h[x].d) break;
    HeapNode s = h[x];
    h[x] = h[t];
    h[t] = s;
    x = t;
  }
}

__global__ void __launch_bounds__(BF_THREADS)
    k_sq8_bruteforce(const int8_t *__restrict__ codes, uint64_t npoints, const int8_t *__restrict__ queries,
                     uint32_t k, int *__restrict__ closest, float *__restrict__ dists, float alpha) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  HeapNode *heap = reinterpret_cast<HeapNode *>(smem_raw);  // [k + 1], 1-based
  HeapNode *list = heap + (k + 1);                          // [BF_CHUNK]
  __shared__ int qw[SQ8_WORDS];
  __shared__ int qq_s;
  __shared__ uint32_t wcount[BF_THREADS / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t qi = blockIdx.x;
  const int8_t *q = queries + (uint64_t)qi * SQ8_CODE;
  if (tid < SQ8_WORDS) qw[tid] = reinterpret_cast<const int *>(q)[tid];
  __syncthreads();
  if (tid == 0) {
    int s = 0;
    for (int w = 0; w < SQ8_WORDS; ++w) s = __dp4a(qw[w], qw[w], s);
    qq_s = s;
  }
  __syncthreads();
  const int qq = qq_s;
  // the first k codes are emplaced unconditionally, in order (bruteforce.h:256-257)
  for (uint32_t base = 0; base < k; base += BF_CHUNK) {
    const uint32_t m = min((uint32_t)BF_CHUNK, k - base);
    for (uint32_t j = tid; j < m; j += BF_THREADS) {
      list[j].d = sq8_dist(qw, qq, codes + (uint64_t)(base + j) * SQ8_CODE);
      list[j].id = (int)(base + j);
    }
    __syncthreads();
    if (tid == 0) {
      for (uint32_t j = 0; j < m; ++j) {
        int now = (int)(base + j) + 1;  // maxPQIFCS::emplace (bruteforce.h:106-113)
        heap[now] = list[j];
        while (now != 1 && heap[now].d > heap[now >> 1].d) {
          HeapNode s = heap[now];
          heap[now] = heap[now >> 1];
          heap[now >> 1] = s;
          now >>= 1;
        }
      }
    }
    __syncthreads();
  }
  // the rest: must_pop_emplace (bruteforce.h:99-105) through the root filter
  for (uint64_t base = k; base < npoints; base += BF_CHUNK) {
    const int root = heap[1].d;
    uint32_t run = 0;
    for (int r = 0; r < BF_CHUNK / BF_THREADS; ++r) {
      const uint64_t p = base + (uint64_t)r * BF_THREADS + tid;
      int d = 0;
      bool keep = false;
      if (p < npoints) {
        d = sq8_dist(qw, qq, codes + p * SQ8_CODE);
        keep = d < root;
      }
      const uint32_t b = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) wcount[warp] = __popc(b);
      __syncthreads();
      uint32_t before = run;
      for (int w = 0; w < warp; ++w) before += wcount[w];
      if (keep) {
        HeapNode nd;
        nd.d = d;
        nd.id = (int)p;
        list[before + __popc(b & ((1u << lane) - 1u))] = nd;
      }
      uint32_t tot = 0;
      for (int w = 0; w < BF_THREADS / 32; ++w) tot += wcount[w];
      run += tot;
      __syncthreads();
    }
    if (tid == 0) {
      for (uint32_t j = 0; j < run; ++j) {
        const HeapNode nd = list[j];
        if (heap[1].d <= nd.d) continue;
        heap[1] = nd;
        heap_push_down(heap, (int)k, 1);
      }
    }
    __syncthreads();
  }
  // closest_points[k - l - 1] = data_[l + 1].id (bruteforce.h:262-264)
  for (uint32_t l = tid; l < k; l += BF_THREADS) {
    closest[(uint64_t)qi * k + (k - l - 1)] = heap[l + 1].id;
    if (dists) dists[(uint64_t)qi * k + (k - l - 1)] = (float)heap[l + 1].d * alpha * alpha;
  }
}

bool is_dev(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

struct Scoped {
  void *p = nullptr;
  ~Scoped() {
    if (p) cudaFree(p);
  }
};

// Device copy of a host buffer (or the pointer itself when it is already a
// 16-byte aligned device pointer; the code rows are read as int4).
int stage_in(const void *src, size_t bytes, Scoped &s, const void **out, cudaStream_t st) {
  if (is_dev(src) && ((uintptr_t)src & 15) == 0) {
    *out = src;
    return FKNN_OK;
  }
  FKNN_CUDA(cudaMalloc(&s.p, bytes ? bytes : 16));
  FKNN_CUDA(cudaMemcpyAsync(s.p, src, bytes, cudaMemcpyDefault, st));
  *out = s.p;
  return FKNN_OK;
}

int stage_out(void *dst, size_t bytes, Scoped &s, void **out) {
  if (is_dev(dst)) {
    *out = dst;
    return FKNN_OK;
  }
  FKNN_CUDA(cudaMalloc(&s.p, bytes ? bytes : 16));
  *out = s.p;
  return FKNN_OK;
}

int ensure_device() {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return FKNN_ENODEV;
  }
  return FKNN_OK;
}

int sq8_encode_impl(const float *vecs, uint64_t n, float alpha, int8_t *codes, bool train, float *alpha_out) {
  if (!vecs || !codes || n == 0) {
    set_error("fknn_sq8: bad arguments");
    return FKNN_EINVAL;
  }
  int rc = ensure_device();
  if (rc) return rc;
  cudaStream_t st = 0;
  Scoped sin, sout, sa;
  const float *d_x;
  int8_t *d_c;
  if ((rc = stage_in(vecs, n * DIM * 4, sin, (const void **)&d_x, st))) return rc;
  if ((rc = stage_out(codes, n * SQ8_CODE, sout, (void **)&d_c))) return rc;
  if (train) {
    FKNN_CUDA(cudaMalloc(&sa.p, 4));
    FKNN_CUDA(cudaMemsetAsync(sa.p, 0, 4, st));
    k_absmax<<<148 * 4, 256, 0, st>>>(d_x, n * DIM, (uint32_t *)sa.p);
    g_launches += 1;
    uint32_t bits = 0;
    FKNN_CUDA(cudaMemcpyAsync(&bits, sa.p, 4, cudaMemcpyDeviceToHost, st));
    FKNN_CUDA(cudaStreamSynchronize(st));
    alpha = bits_f32(bits);
    if (alpha_out) *alpha_out = alpha;
  }
  if (!(alpha > 0.f) || !(alpha <= 3.0e38f)) {
    set_error("fknn_sq8: alpha must be positive and finite (all-zero or non-finite training data?)");
    return FKNN_EINVAL;
  }
  k_sq8_encode<<<148 * 8, 256, 0, st>>>(d_x, n, alpha, d_c);
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  if (d_c != codes) FKNN_CUDA(cudaMemcpyAsync(codes, d_c, n * SQ8_CODE, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  return FKNN_OK;
}

int sq8_bf_impl(size_t k, int *closest, float *dists, size_t npoints, const char *codes_in, float alpha,
                size_t nqueries, const int8_t *queries_in) {
  if (!closest || !codes_in || !queries_in || k == 0 || k > npoints || k > (size_t)BF_KMAX || nqueries == 0 ||
      npoints >= (1ull << 31)) {
    set_error("fknn_sq8_bruteforce: need 1 <= k <= npoints, k <= 2048, nqueries >= 1, npoints < 2^31");
    return FKNN_EINVAL;
  }
  int rc = ensure_device();
  if (rc) return rc;
  cudaStream_t st = 0;
  Scoped sc, sq, si, sd;
  const int8_t *d_codes, *d_q;
  int *d_ids;
  float *d_d = nullptr;
  if ((rc = stage_in(codes_in, npoints * SQ8_CODE, sc, (const void **)&d_codes, st))) return rc;
  if ((rc = stage_in(queries_in, nqueries * SQ8_CODE, sq, (const void **)&d_q, st))) return rc;
  if ((rc = stage_out(closest, nqueries * k * 4, si, (void **)&d_ids))) return rc;
  if (dists)
    if ((rc = stage_out(dists, nqueries * k * 4, sd, (void **)&d_d))) return rc;
  const size_t smem = (k + 1 + BF_CHUNK) * sizeof(HeapNode);
  FKNN_CUDA(cudaFuncSetAttribute(k_sq8_bruteforce, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_sq8_bruteforce<<<(unsigned)nqueries, BF_THREADS, smem, st>>>(d_codes, npoints, d_q, (uint32_t)k, d_ids, d_d,
                                                                 alpha);
  g_launches += 1;
  FKNN_CUDA(cudaGetLastError());
  if (d_ids != closest) FKNN_CUDA(cudaMemcpyAsync(closest, d_ids, nqueries * k * 4, cudaMemcpyDeviceToHost, st));
  if (dists && d_d != dists) FKNN_CUDA(cudaMemcpyAsync(dists, d_d, nqueries * k * 4, cudaMemcpyDeviceToHost, st));
  FKNN_CUDA(cudaStreamSynchronize(st));
  return FKNN_OK;
}

}  // namespace

void launch_sq8_encode(const float *d_x, uint64_t n, float alpha, int8_t *d_codes, cudaStream_t st) {
  k_sq8_encode<<<148 * 8, 256, 0, st>>>(d_x, n, alpha, d_codes);
  g_launches += 1;
}

}  // namespace fknn

using namespace fknn;

extern "C" {

int fknn_sq8_sym_train(const float *vecs, uint64_t n, float *alpha, int8_t *codes) {
  g_launches = 0;
  if (!alpha) {
    set_error("fknn_sq8_sym_train: alpha is NULL");
    return FKNN_EINVAL;
  }
  return sq8_encode_impl(vecs, n, 0.f, codes, true, alpha);
}

int fknn_sq8_sym_encode(const float *vecs, uint64_t n, float alpha, int8_t *codes) {
  g_launches = 0;
  return sq8_encode_impl(vecs, n, alpha, codes, false, nullptr);
}

int fknn_sq8_bruteforce(size_t dim, size_t k, int *closest_points, size_t npoints, const char *codes_in, float alpha,
                        size_t nqueries, const int8_t *queries_in) {
  (void)dim;
  g_launches = 0;
  return sq8_bf_impl(k, closest_points, nullptr, npoints, codes_in, alpha, nqueries, queries_in);
}

int fknn_sq8_bruteforce_subgraph(size_t dim, size_t k, int *closest_points, float *distances, size_t npoints,
                                 const char *codes_in, float alpha, size_t nqueries, const int8_t *queries_in) {
  (void)dim;
  g_launches = 0;
  if (!distances) {
    set_error("fknn_sq8_bruteforce_subgraph: distances is NULL");
    return FKNN_EINVAL;
  }
  return sq8_bf_impl(k, closest_points, distances, npoints, codes_in, alpha, nqueries, queries_in);
}

}  // extern "C"
