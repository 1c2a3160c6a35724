// Request loop with continuous batching over one resident index.
//
// The reference answers queries in one offline batch (baseline.cpp:150,
// HybridGraph::BatchSearch); this loop serves a stream of them.  Requests
// are queued per query type (the reference's four filter types), and
// whenever a slot frees up the scheduler gives it the oldest type's waiting
// requests, up to max_batch, provided the device scratch the slots hold
// fits in the HBM budget.  A batch that runs over the budget releases its
// slot's scratch and lowers its query type's batch size.  Each
// slot is a search view of the index (shared vectors, codes and row
// orders; its own scratch) driven by its own host thread on its own
// stream, so one batch's kernels run while another batch plans or copies.
// A request's result does not depend on the batch it rode in: every
// search form computes each query's answer from that query and the index
// alone.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fknn_internal.cuh"

namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Request {
  float q[fknn::DIM];
  float meta[4];
  uint32_t *ids;
  float *dists;
  int64_t t_arrive;
  int status;
  bool done;
};

struct Slot {
  fknn_index *view = nullptr;
  cudaStream_t stream = nullptr;
  float *h_q = nullptr, *h_m = nullptr, *h_d = nullptr;  // pinned staging, max_batch rows
  uint32_t *h_ids = nullptr;
  std::vector<uint64_t> batch;  // tickets of the assigned batch
  bool busy = false, has_work = false;
  uint64_t footprint = 0;       // device bytes of the view's scratch
  std::thread th;
};

}  // namespace

struct fknn_server {
  fknn_index *idx = nullptr;
  fknn_server_opts o{};
  fknn_search_opts so{};
  uint64_t budget = 0;
  std::mutex mu;
  std::condition_variable cv_sched, cv_slot, cv_done;
  std::deque<Request> reqs;  // tickets [base, base + reqs.size())
  uint64_t base = 0, next = 0;
  std::deque<uint64_t> queue[4];
  std::unordered_map<uint64_t, int> failed;
  std::vector<Slot *> slots;
  std::thread sched;
  bool stop = false;
  uint32_t cap[4] = {0, 0, 0, 0};  // admitted batch size per query type
  // statistics since the last reset
  std::vector<float> lat_ms;
  uint64_t submitted = 0, completed = 0, nfailed = 0, batches = 0, admission_waits = 0, batch_queries = 0,
           trims = 0;
  uint32_t max_batch_seen = 0;
  int64_t first_arrival = INT64_MAX, last_done = 0;
  std::string last_error;
};

namespace {

using fknn::DIM;

bool valid_query(const float *q, const float *m) {
  for (int d = 0; d < DIM; ++d)
    if (!(std::fabs(q[d]) <= 1e15f)) return false;
  const float t = m[0];
  if (!(t == 0.f || t == 1.f || t == 2.f || t == 3.f)) return false;
  if ((t == 1.f || t == 3.f) && !(std::fabs(m[1]) < 2147483648.f)) return false;
  if ((t == 2.f || t == 3.f) && (m[2] != m[2] || m[3] != m[3])) return false;
  return true;
}

// Queries of type t a slot may take now: a batch starts only while the
// scratch the slots hold fits in the budget, and at most the type's batch
// cap, which shrinks when a batch of that type ran over the budget.
uint32_t admit_limit(fknn_server *s, int t) {
  uint64_t held = 0;
  for (Slot *x : s->slots) held += x->footprint;
  if (s->budget && held > s->budget) return 0;
  return s->cap[t];
}

void scheduler(fknn_server *s) {
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    Slot *free_slot = nullptr;
    for (Slot *x : s->slots)
      if (!x->busy) {
        free_slot = x;
        break;
      }
    int t = -1;
    int64_t oldest = INT64_MAX;
    for (int i = 0; i < 4; ++i)
      if (!s->queue[i].empty()) {
        const int64_t a = s->reqs[s->queue[i].front() - s->base].t_arrive;
        if (a < oldest) {
          oldest = a;
          t = i;
        }
      }
    if (!free_slot || t < 0) {
      s->cv_sched.wait(lk);
      continue;
    }
    // optional linger for a fuller batch while other slots keep the device busy
    if (s->o.max_wait_us && s->queue[t].size() < s->o.max_batch) {
      bool any_busy = false;
      for (Slot *x : s->slots) any_busy |= x->busy;
      const int64_t due = oldest + (int64_t)s->o.max_wait_us * 1000;
      if (any_busy && now_ns() < due) {
        s->cv_sched.wait_for(lk, std::chrono::nanoseconds(due - now_ns()));
        continue;
      }
    }
    const uint32_t take = std::min<uint32_t>((uint32_t)s->queue[t].size(), admit_limit(s, t));
    if (take == 0) {  // the budget admits nothing until a slot's batch ends
      ++s->admission_waits;
      s->cv_sched.wait(lk);
      continue;
    }
    free_slot->batch.assign(s->queue[t].begin(), s->queue[t].begin() + take);
    s->queue[t].erase(s->queue[t].begin(), s->queue[t].begin() + take);
    free_slot->busy = true;
    free_slot->has_work = true;
    s->cv_slot.notify_all();
  }
}

void worker(fknn_server *s, Slot *slot) {
  const uint32_t k = s->o.k;
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv_slot.wait(lk, [&] { return slot->has_work || s->stop; });
    if (!slot->has_work) return;
    slot->has_work = false;
    const std::vector<uint64_t> batch = slot->batch;
    std::vector<Request *> rs(batch.size());
    for (size_t i = 0; i < batch.size(); ++i) rs[i] = &s->reqs[batch[i] - s->base];
    lk.unlock();
    const uint32_t nb = (uint32_t)batch.size();
    for (uint32_t i = 0; i < nb; ++i) {
      std::memcpy(slot->h_q + (size_t)i * DIM, rs[i]->q, DIM * sizeof(float));
      std::memcpy(slot->h_m + (size_t)i * 4, rs[i]->meta, 4 * sizeof(float));
    }
    const int rc = fknn_search_ex(slot->view, slot->h_q, slot->h_m, nb, k, &s->so, slot->h_ids, slot->h_d,
                                  slot->stream, nullptr);
    std::string err = rc ? std::string(fknn_last_error()) : std::string();
    if (rc == 0)
      for (uint32_t i = 0; i < nb; ++i) {
        if (rs[i]->ids) std::memcpy(rs[i]->ids, slot->h_ids + (size_t)i * k, k * sizeof(uint32_t));
        if (rs[i]->dists) std::memcpy(rs[i]->dists, slot->h_d + (size_t)i * k, k * sizeof(float));
      }
    const int64_t t_done = now_ns();
    uint64_t fp = fknn::scratch_bytes(slot->view);
    lk.lock();
    const int t = (int)rs[0]->meta[0];
    uint64_t others = 0;
    for (Slot *x : s->slots)
      if (x != slot) others += x->footprint;
    if (s->budget && others + fp > s->budget) {
      // ran over: release this slot's scratch and admit smaller batches of this type
      const uint64_t room = s->budget > others ? s->budget - others : 0;
      s->cap[t] = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(nb - (nb > 1), (uint64_t)nb * room / fp));
      ++s->trims;
      lk.unlock();
      fknn::trim_scratch(slot->view);
      fp = fknn::scratch_bytes(slot->view);
      lk.lock();
    }
    slot->footprint = fp;
    for (Request *r : rs) {
      r->status = rc;
      r->done = true;
      s->lat_ms.push_back((float)((t_done - r->t_arrive) * 1e-6));
      s->first_arrival = std::min(s->first_arrival, r->t_arrive);
    }
    if (rc) {
      s->nfailed += nb;
      s->last_error = err;
      for (uint64_t tk : batch) s->failed[tk] = rc;
    }
    s->completed += nb;
    s->batches += 1;
    s->batch_queries += nb;
    s->max_batch_seen = std::max(s->max_batch_seen, nb);
    s->last_done = std::max(s->last_done, t_done);
    while (!s->reqs.empty() && s->reqs.front().done) {
      s->reqs.pop_front();
      ++s->base;
    }
    slot->busy = false;
    s->cv_sched.notify_all();
    s->cv_done.notify_all();
  }
}

void destroy_server(fknn_server *s) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_sched.notify_all();
  s->cv_slot.notify_all();
  if (s->sched.joinable()) s->sched.join();
  for (Slot *x : s->slots) {
    if (x->th.joinable()) x->th.join();
    if (x->stream) cudaStreamDestroy(x->stream);
    if (x->h_q) cudaFreeHost(x->h_q);
    if (x->h_m) cudaFreeHost(x->h_m);
    if (x->h_ids) cudaFreeHost(x->h_ids);
    if (x->h_d) cudaFreeHost(x->h_d);
    if (x->view) fknn::destroy_index(x->view);
    delete x;
  }
  delete s;
}

}  // namespace

extern "C" {

int64_t fknn_server_now_ns(void) { return now_ns(); }

int fknn_server_create(fknn_index *idx, const fknn_server_opts *opts, fknn_server **out) {
  using fknn::set_error;
  if (!idx || !out) {
    set_error("fknn_server_create: NULL argument");
    return FKNN_EINVAL;
  }
  *out = nullptr;
  fknn_server_opts o{};
  if (opts) o = *opts;
  if (o.k == 0) o.k = 100;
  if (o.max_batch == 0) o.max_batch = 4096;
  if (o.slots == 0) o.slots = 3;
  if (o.k > 128 || o.slots > 16 || o.max_batch > (1u << 20)) {
    set_error("fknn_server_create: need k <= 128, slots <= 16, max_batch <= 2^20");
    return FKNN_EINVAL;
  }
  if (o.mode != FKNN_MODE_EXACT_FP32 && o.mode != FKNN_MODE_BF16_RERANK && o.mode != FKNN_MODE_FP8_RERANK) {
    set_error("fknn_server_create: unknown mode");
    return FKNN_EINVAL;
  }
  if ((o.mode == FKNN_MODE_BF16_RERANK && !idx->bf16_blocks[0]) ||
      (o.mode == FKNN_MODE_FP8_RERANK && !idx->fp8_blocks[0])) {
    set_error("fknn_server_create: the index was created without that mode's copies");
    return FKNN_EUNSUPPORTED;
  }
  fknn_server *s = new (std::nothrow) fknn_server();
  if (!s) return FKNN_ENOMEM;
  s->idx = idx;
  s->o = o;
  s->so.mode = o.mode;
  s->so.kprime = o.kprime;
  for (int t = 0; t < 4; ++t) s->cap[t] = o.max_batch;
  int rc = FKNN_OK;
  cudaError_t e = cudaSetDevice(idx->device);
  if (e != cudaSuccess) rc = fknn::cuda_fail(e, "cudaSetDevice");
  s->budget = o.hbm_budget;
  if (!rc && s->budget == 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) s->budget = fr / 2;
  }
  for (uint32_t i = 0; i < o.slots && !rc; ++i) {
    Slot *x = new (std::nothrow) Slot();
    if (!x) {
      rc = FKNN_ENOMEM;
      break;
    }
    s->slots.push_back(x);
    rc = fknn::make_index_view(idx, &x->view);
    if (rc) break;
    e = cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking);
    const size_t mb = o.max_batch;
    if (e == cudaSuccess) e = cudaMallocHost(&x->h_q, mb * DIM * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&x->h_m, mb * 4 * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&x->h_ids, mb * o.k * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMallocHost(&x->h_d, mb * o.k * sizeof(float));
    if (e != cudaSuccess) rc = fknn::cuda_fail(e, "fknn_server_create");
  }
  if (rc) {
    destroy_server(s);
    return rc;
  }
  for (Slot *x : s->slots) x->th = std::thread(worker, s, x);
  s->sched = std::thread(scheduler, s);
  *out = s;
  return FKNN_OK;
}

int fknn_server_submit(fknn_server *s, const float *qvecs, const float *metas, uint32_t nreq,
                       const int64_t *arrival_ns, uint32_t *ids, float *dists, uint64_t *first_ticket) {
  using fknn::set_error;
  if (!s || (nreq && (!qvecs || !metas))) {
    set_error("fknn_server_submit: NULL argument");
    return FKNN_EINVAL;
  }
  for (uint32_t i = 0; i < nreq; ++i)
    if (!valid_query(qvecs + (size_t)i * DIM, metas + (size_t)i * 4)) {
      set_error("fknn_server_submit: request " + std::to_string(i) +
                " has a type outside {0,1,2,3}, a category outside int32, a NaN window bound or a non-finite vector");
      return FKNN_EINVAL;
    }
  const int64_t t_now = now_ns();
  std::lock_guard<std::mutex> lk(s->mu);
  if (first_ticket) *first_ticket = s->next;
  for (uint32_t i = 0; i < nreq; ++i) {
    s->reqs.emplace_back();
    Request &r = s->reqs.back();
    std::memcpy(r.q, qvecs + (size_t)i * DIM, sizeof(r.q));
    std::memcpy(r.meta, metas + (size_t)i * 4, sizeof(r.meta));
    r.ids = ids ? ids + (size_t)i * s->o.k : nullptr;
    r.dists = dists ? dists + (size_t)i * s->o.k : nullptr;
    r.t_arrive = arrival_ns ? arrival_ns[i] : t_now;
    r.status = 0;
    r.done = false;
    s->queue[(int)r.meta[0]].push_back(s->next++);
  }
  s->submitted += nreq;
  s->cv_sched.notify_all();
  return FKNN_OK;
}

int fknn_server_wait(fknn_server *s, uint64_t ticket, int timeout_ms) {
  if (!s) return FKNN_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  if (ticket >= s->next) {
    fknn::set_error("fknn_server_wait: unknown ticket");
    return FKNN_EINVAL;
  }
  auto done = [&] { return ticket < s->base || s->reqs[ticket - s->base].done; };
  if (timeout_ms < 0) s->cv_done.wait(lk, done);
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
    fknn::set_error("fknn_server_wait: timed out");
    return FKNN_ETIMEOUT;
  }
  auto it = s->failed.find(ticket);
  if (it != s->failed.end()) {
    fknn::set_error(s->last_error);
    return it->second;
  }
  return FKNN_OK;
}

int fknn_server_drain(fknn_server *s, int timeout_ms) {
  if (!s) return FKNN_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  auto done = [&] { return s->base == s->next; };
  if (timeout_ms < 0) s->cv_done.wait(lk, done);
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
    fknn::set_error("fknn_server_drain: timed out");
    return FKNN_ETIMEOUT;
  }
  if (!s->failed.empty()) {
    fknn::set_error(s->last_error);
    return s->failed.begin()->second;
  }
  return FKNN_OK;
}

int fknn_server_get_stats(fknn_server *s, fknn_server_stats *out, int reset) {
  if (!s || !out) return FKNN_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->failed = s->nfailed;
  out->batches = s->batches;
  out->admission_waits = s->admission_waits;
  out->budget_trims = s->trims;
  for (Slot *x : s->slots) out->scratch_bytes += x->footprint;
  out->budget_bytes = s->budget;
  out->max_batch_seen = s->max_batch_seen;
  out->mean_batch = s->batches ? (float)s->batch_queries / (float)s->batches : 0.f;
  if (!s->lat_ms.empty()) {
    std::vector<float> v = s->lat_ms;
    auto pct = [&](double p) {
      const size_t i = std::min(v.size() - 1, (size_t)(p * (double)(v.size() - 1) + 0.5));
      std::nth_element(v.begin(), v.begin() + i, v.end());
      return v[i];
    };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->max_ms = *std::max_element(v.begin(), v.end());
    double sum = 0;
    for (float x : v) sum += x;
    out->mean_ms = (float)(sum / v.size());
    out->span_s = (double)(s->last_done - s->first_arrival) * 1e-9;
    out->qps = out->span_s > 0 ? (double)v.size() / out->span_s : 0.0;
  }
  if (reset) {
    s->lat_ms.clear();
    s->submitted = s->completed = s->nfailed = s->batches = s->admission_waits = s->batch_queries = s->trims = 0;
    s->max_batch_seen = 0;
    s->first_arrival = INT64_MAX;
    s->last_done = 0;
  }
  return FKNN_OK;
}

int fknn_server_destroy(fknn_server *s) {
  if (!s) return FKNN_OK;
  fknn_server_drain(s, -1);
  destroy_server(s);
  return FKNN_OK;
}

}  // extern "C"
