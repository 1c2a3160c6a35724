// The contest's binary files through the C ABI:
//   base    u32 N, then N rows [label f32, ts f32, 100 x f32]   ReadBase        utils.h:257-276
//   queries u32 Q, then Q rows [type, v, l, r, 100 x f32]        ReadQuery       utils.h:550-566
//   knn     Q x k u32, no header                                 SaveKNN         io.h:22-33
//   gt      u32 Q, then Q x k u32                                ReadGroundTruth utils.h:194-221
// plus the query order of ReadSortedQuery (utils.h:491-548) and the ingest
// of a base file straight into a resident index: the rows stream from the
// file through two pinned buffers to the device, where a kernel splits them
// into the index's columns, and the row orders that ReadSortedBaseTimestamp
// (utils.h:352-479) builds with host sorts are built by the index's radix
// sorts on the GPU.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "device_util.cuh"

namespace fknn {

namespace {

constexpr int ROW_F = DIM + 2;           // floats per base row
constexpr int QROW_F = DIM + 4;          // floats per query row
constexpr uint64_t INGEST_ROWS = 1 << 16;  // rows per streamed chunk (26.7 MB)

struct File {
  FILE *f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

int open_counted(const char *path, const char *who, File &F, uint32_t *n, uint64_t row_bytes) {
  if (!path) {
    set_error(std::string(who) + ": path is NULL");
    return FKNN_EINVAL;
  }
  F.f = fopen(path, "rb");
  if (!F.f) {
    set_error(std::string(who) + ": cannot open " + path);
    return FKNN_EINVAL;
  }
  if (fread(n, 4, 1, F.f) != 1) {
    set_error(std::string(who) + ": no header in " + path);
    return FKNN_EINVAL;
  }
  if (fseeko(F.f, 0, SEEK_END) != 0) {
    set_error(std::string(who) + ": cannot seek in " + path);
    return FKNN_EINVAL;
  }
  const uint64_t size = (uint64_t)ftello(F.f);
  if (size < 4 + (uint64_t)*n * row_bytes) {
    set_error(std::string(who) + ": " + path + " holds fewer rows than its header says");
    return FKNN_EINVAL;
  }
  fseeko(F.f, 4, SEEK_SET);
  return FKNN_OK;
}

__global__ void k_split_rows(const float *__restrict__ rows, uint64_t nrows, float *__restrict__ vecs,
                             float *__restrict__ labels, float *__restrict__ ts) {
  const uint64_t total = nrows * ROW_F;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i / ROW_F;
    const uint32_t c = (uint32_t)(i - r * ROW_F);
    const float v = rows[i];
    if (c == 0) labels[r] = v;
    else if (c == 1) ts[r] = v;
    else vecs[r * DIM + (c - 2)] = v;
  }
}

// Streams the base rows of an open file into the index's device columns.
int ingest_rows(fknn_index *idx, FILE *f, cudaStream_t st) {
  const uint64_t n = idx->n;
  int rc;
  if ((rc = alloc_index_columns(idx))) return rc;
  const size_t chunk_bytes = (size_t)INGEST_ROWS * ROW_F * sizeof(float);
  float *h[2] = {nullptr, nullptr}, *d = nullptr;
  cudaEvent_t done[2] = {nullptr, nullptr};
  auto cleanup = [&]() {
    for (int b = 0; b < 2; ++b) {
      if (done[b]) cudaEventDestroy(done[b]);
      if (h[b]) cudaFreeHost(h[b]);
    }
    if (d) cudaFree(d);
  };
  cudaError_t e = cudaSuccess;
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
    e = cudaMallocHost(&h[b], chunk_bytes);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaMalloc(&d, 2 * chunk_bytes);
  if (e != cudaSuccess) {
    cleanup();
    return cuda_fail(e, "fknn_index_create_from_file: staging buffers");
  }
  uint64_t r0 = 0;
  for (int b = 0; r0 < n; b ^= 1) {
    const uint64_t m = std::min<uint64_t>(INGEST_ROWS, n - r0);
    // the pinned buffer is free once its previous copy has finished
    if ((e = cudaEventSynchronize(done[b])) != cudaSuccess) break;
    if (fread(h[b], (size_t)m * ROW_F * sizeof(float), 1, f) != 1) {
      cleanup();
      set_error("fknn_index_create_from_file: short read");
      return FKNN_EINVAL;
    }
    float *db = d + (size_t)b * INGEST_ROWS * ROW_F;
    if ((e = cudaMemcpyAsync(db, h[b], (size_t)m * ROW_F * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
      break;
    if ((e = cudaEventRecord(done[b], st)) != cudaSuccess) break;
    const unsigned grid = (unsigned)std::min<uint64_t>((m * ROW_F + 255) / 256, 148 * 8);
    k_split_rows<<<grid, 256, 0, st>>>(db, m, idx->vecs + r0 * DIM, idx->labels_f + r0, idx->ts_f + r0);
    g_launches += 1;
    r0 += m;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cleanup();
  if (e != cudaSuccess) return cuda_fail(e, "fknn_index_create_from_file: streaming the rows");
  return build_index_from_columns(idx, st);
}

}  // namespace

}  // namespace fknn

using namespace fknn;

extern "C" {

int fknn_read_base_file(const char *path, uint64_t *n, float *vecs, float *labels, float *ts) {
  if (!n) {
    set_error("fknn_read_base_file: n is NULL");
    return FKNN_EINVAL;
  }
  File F;
  uint32_t cnt = 0;
  int rc = open_counted(path, "fknn_read_base_file", F, &cnt, ROW_F * sizeof(float));
  if (rc) return rc;
  *n = cnt;
  if (!vecs && !labels && !ts) return FKNN_OK;  // size query
  if (!vecs || !labels || !ts) {
    set_error("fknn_read_base_file: vecs, labels and ts must all be given (or all NULL)");
    return FKNN_EINVAL;
  }
  std::vector<float> buf((size_t)std::min<uint64_t>(cnt, INGEST_ROWS) * ROW_F);
  for (uint64_t r0 = 0; r0 < cnt;) {
    const uint64_t m = std::min<uint64_t>(INGEST_ROWS, cnt - r0);
    if (fread(buf.data(), (size_t)m * ROW_F * sizeof(float), 1, F.f) != 1) {
      set_error("fknn_read_base_file: short read");
      return FKNN_EINVAL;
    }
    for (uint64_t i = 0; i < m; ++i) {
      const float *row = buf.data() + i * ROW_F;
      labels[r0 + i] = row[0];
      ts[r0 + i] = row[1];
      std::memcpy(vecs + (r0 + i) * DIM, row + 2, DIM * sizeof(float));
    }
    r0 += m;
  }
  return FKNN_OK;
}

int fknn_read_query_file(const char *path, uint32_t *nq, float *qvecs, float *metas) {
  if (!nq) {
    set_error("fknn_read_query_file: nq is NULL");
    return FKNN_EINVAL;
  }
  File F;
  uint32_t cnt = 0;
  int rc = open_counted(path, "fknn_read_query_file", F, &cnt, QROW_F * sizeof(float));
  if (rc) return rc;
  *nq = cnt;
  if (!qvecs && !metas) return FKNN_OK;
  if (!qvecs || !metas) {
    set_error("fknn_read_query_file: qvecs and metas must both be given (or both NULL)");
    return FKNN_EINVAL;
  }
  std::vector<float> row(QROW_F);
  for (uint32_t i = 0; i < cnt; ++i) {
    if (fread(row.data(), sizeof(float) * QROW_F, 1, F.f) != 1) {
      set_error("fknn_read_query_file: short read");
      return FKNN_EINVAL;
    }
    std::memcpy(metas + (size_t)i * 4, row.data(), 4 * sizeof(float));
    std::memcpy(qvecs + (size_t)i * DIM, row.data() + 4, DIM * sizeof(float));
  }
  return FKNN_OK;
}

int fknn_sorted_query_order(const float *metas, uint32_t nq, uint32_t *sorted_ids) {
  if ((!metas || !sorted_ids) && nq) {
    set_error("fknn_sorted_query_order: NULL argument");
    return FKNN_EINVAL;
  }
  std::iota(sorted_ids, sorted_ids + nq, 0u);
  // (type as uint32, v as int32, l, r) ascending; equal keys keep their order
  std::stable_sort(sorted_ids, sorted_ids + nq, [&](uint32_t a, uint32_t b) {
    const float *ma = metas + (size_t)a * 4, *mb = metas + (size_t)b * 4;
    const uint32_t ta = (uint32_t)ma[0], tb = (uint32_t)mb[0];
    if (ta != tb) return ta < tb;
    const int32_t ca = (int32_t)ma[1], cb = (int32_t)mb[1];
    if (ca != cb) return ca < cb;
    if (ma[2] != mb[2]) return ma[2] < mb[2];
    return ma[3] < mb[3];
  });
  return FKNN_OK;
}

int fknn_save_knn(const char *path, const uint32_t *ids, uint32_t nq, uint32_t k) {
  if (!path || (!ids && nq) || k == 0) {
    set_error("fknn_save_knn: NULL argument or k = 0");
    return FKNN_EINVAL;
  }
  FILE *f = fopen(path, "wb");
  if (!f) {
    set_error(std::string("fknn_save_knn: cannot create ") + path);
    return FKNN_EINVAL;
  }
  const size_t w = nq ? fwrite(ids, (size_t)nq * k * sizeof(uint32_t), 1, f) : 1;
  const int c = fclose(f);
  if (w != 1 || c != 0) {
    set_error(std::string("fknn_save_knn: write to ") + path + " failed");
    return FKNN_EINVAL;
  }
  return FKNN_OK;
}

int fknn_read_groundtruth(const char *path, uint32_t k, uint32_t *nq, uint32_t *ids) {
  if (!nq || k == 0) {
    set_error("fknn_read_groundtruth: nq is NULL or k = 0");
    return FKNN_EINVAL;
  }
  File F;
  uint32_t cnt = 0;
  int rc = open_counted(path, "fknn_read_groundtruth", F, &cnt, (uint64_t)k * sizeof(uint32_t));
  if (rc) return rc;
  *nq = cnt;
  if (!ids || !cnt) return FKNN_OK;
  if (fread(ids, (size_t)cnt * k * sizeof(uint32_t), 1, F.f) != 1) {
    set_error("fknn_read_groundtruth: short read");
    return FKNN_EINVAL;
  }
  return FKNN_OK;
}

int fknn_index_create_from_file(const char *path, const fknn_index_opts *opts, fknn_index **out) {
  if (!out) {
    set_error("fknn_index_create_from_file: out is NULL");
    return FKNN_EINVAL;
  }
  *out = nullptr;
  g_launches = 0;
  File F;
  uint32_t cnt = 0;
  int rc = open_counted(path, "fknn_index_create_from_file", F, &cnt, ROW_F * sizeof(float));
  if (rc) return rc;
  return create_index(cnt, opts, [&](fknn_index *idx, cudaStream_t st) { return ingest_rows(idx, F.f, st); }, out);
}

}  // extern "C"
