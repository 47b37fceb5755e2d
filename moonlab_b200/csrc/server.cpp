// server.cpp -- continuous-batching request loop on one GPU.
//
// Requests (a circuit, a dtype, a shot count and a seed) queue on the host;
// worker threads admit them in arrival order as soon as a worker slot and
// HBM budget are free, so requests that arrive while others run start
// without waiting for a batch boundary, and their kernels overlap on the
// device (each request runs on its own state's stream).  States are pooled
// per (qubits, dtype): a finished request's state is reset and reused, so
// the steady state does no cudaMalloc / cudaFree (cudaFree would stall the
// whole device).  Pooled states count against the budget; a request of a
// new size class evicts idle pooled states when it has to.
//
// A request's shots follow moonlab_qgtl_execute (moonlab_qgtl_backend.c:
// 218-240): uniforms from xorshift64(seed) (a zero seed takes the clock),
// each shot measurement_all_qubits(u) on the circuit's output state; for
// complex128 the outcomes are bit-identical to the reference's.  A request's
// result does not depend on what else runs: its kernels read and write only
// its own state and every reduction has a fixed order.
//
// Small requests (<= 12 qubits complex128, <= 13 complex64) need no pooled
// state: a worker that admits one also takes every other small request of
// the same dtype waiting in the queue and runs them all in one launch, one
// CTA per circuit with the state in shared memory (kernels_small.cu), on its
// own stream.
//
// Pooled states keep a plan cache: a request whose circuit shape (gate
// kinds and qubits, not angles) ran before on that state skips planning and
// replays the passes' launches as one CUDA graph.
//
// A large state's tile passes fill every SM for the length of a pass, so
// each pooled state gets its own stream with a priority by size class
// (smaller states higher): whenever SMs free up, the block scheduler
// starts the small requests' kernels first, and a short request that
// arrives behind a long one finishes long before it.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <ctime>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "moonlab_b200.h"
#include "mlb_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

constexpr size_t kStateOverhead = 1 << 20;  // per-state scratch and sampling buffers, bounded
constexpr size_t kMaxSmallBatch = 1024;     // small requests per launch

struct Request {
  uint64_t ticket = 0;
  uint32_t n = 0;
  int dtype = MLB_C128;
  std::vector<mlb_gate_t> gates;
  uint32_t shots = 0;
  uint64_t seed = 0;
  int status = 1;  // 1 pending, 2 running, else final mlb_status_t (written under mu)
  int result = 0;  // a small batch's outcome for this request, published as status under mu
  std::vector<uint64_t> outcomes;
  double t_submit = 0, t_admit = 0, t_done = 0;
  size_t bytes = 0;
};

size_t state_bytes(uint32_t n, int dtype) {
  return ((size_t)(dtype == MLB_C128 ? 16 : 8) << n) + kStateOverhead;
}

uint64_t xorshift64(uint64_t& s) {  // moonlab_qgtl_backend.c:159-167
  uint64_t x = s;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  s = x;
  return x;
}

}  // namespace

struct mlb_server {
  int device = 0;
  size_t budget = 0;
  int num_workers = 1;
  double starvation_s = 0.5;
  Clock::time_point t0;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::unordered_map<uint64_t, Request*> by_ticket;
  std::map<std::pair<uint32_t, int>, std::vector<mlb_state_t*>> idle;  // pooled, free
  std::unordered_map<mlb_state_t*, cudaStream_t> streams;  // the server's stream of each state
  int prio_least = 0, prio_greatest = 0;
  size_t reserved = 0;  // bytes of all states held (running + idle) and reservations
  int running = 0;
  bool stopping = false;
  uint64_t next_ticket = 1;
  mlb_server_stats_t st{};
  std::vector<std::thread> threads;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

  // Under mu: pick the next request to admit.  *state gets an idle pooled
  // state when one fits; otherwise the request's bytes are reserved and
  // *evict lists idle states to free first.  First fit in arrival order,
  // except that a request waiting longer than starvation_s blocks later ones.
  static bool is_small(const Request* r) { return (int)r->n <= mlb::small_max_qubits(r->dtype); }

  Request* pick(mlb_state_t** state, std::vector<mlb_state_t*>* evict) {
    const double t = now();
    for (auto it = pending.begin(); it != pending.end(); ++it) {
      Request* r = *it;
      if (is_small(r)) {  // no device state of its own
        *state = nullptr;
        pending.erase(it);
        return r;
      }
      auto key = std::make_pair(r->n, r->dtype);
      auto pit = idle.find(key);
      if (pit != idle.end() && !pit->second.empty()) {
        *state = pit->second.back();
        pit->second.pop_back();
        pending.erase(it);
        return r;
      }
      size_t free_bytes = budget > reserved ? budget - reserved : 0;
      if (r->bytes <= free_bytes) {
        reserved += r->bytes;
        *state = nullptr;
        pending.erase(it);
        return r;
      }
      // evict idle states of other classes if that makes room
      size_t idle_bytes = 0;
      for (auto& kv : idle) idle_bytes += kv.second.size() * state_bytes(kv.first.first, kv.first.second);
      if (r->bytes <= free_bytes + idle_bytes) {
        for (auto& kv : idle) {
          while (!kv.second.empty() && r->bytes > free_bytes) {
            evict->push_back(kv.second.back());
            kv.second.pop_back();
            const size_t b = state_bytes(kv.first.first, kv.first.second);
            reserved -= b;
            free_bytes += b;
          }
        }
        reserved += r->bytes;
        *state = nullptr;
        pending.erase(it);
        return r;
      }
      if (t - r->t_submit > starvation_s) return nullptr;  // hold the line for it
    }
    return nullptr;
  }

  // Stream priority of a size class: up to 16 qubits the highest, one level
  // down per 3 qubits above that.
  int priority(uint32_t n) const {
    int level = n <= 16 ? 0 : (int)(n - 14) / 3;
    int p = prio_greatest + level;
    return p > prio_least ? prio_least : p;
  }

  int new_state(uint32_t n, int dtype, mlb_state_t** out) {
    int rc = mlb_state_create(n, dtype, device, out);
    if (rc) return rc;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, priority(n));
    if (e == cudaSuccess) rc = mlb_state_set_stream(*out, (void*)st);
    if (e == cudaSuccess && !rc) rc = mlb_state_set_plan_cache(*out, 8);  // repeated circuit shapes
    if (e != cudaSuccess || rc) {
      if (st) cudaStreamDestroy(st);
      mlb_state_free(*out);
      *out = nullptr;
      return e != cudaSuccess ? mlb::record_error(MLB_ERR_DRIVER, "stream creation failed") : rc;
    }
    std::lock_guard<std::mutex> lk(mu);
    streams[*out] = st;
    return MLB_OK;
  }

  // Frees a state and the server's stream of it (not under mu).
  void free_state(mlb_state_t* s) {
    cudaStream_t st = nullptr;
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = streams.find(s);
      if (it != streams.end()) {
        st = it->second;
        streams.erase(it);
      }
    }
    mlb_state_free(s);  // synchronises the state's stream first
    if (st) cudaStreamDestroy(st);
  }

  // Device buffers of one worker's small batches (grow only).
  struct SmallBufs {
    cudaStream_t stream = nullptr;
    mlb::SmallItem* items = nullptr;
    mlb_op_t* ops = nullptr;
    double* uni = nullptr;
    unsigned long long* out = nullptr;
    size_t cap_items = 0, cap_ops = 0, cap_uni = 0, cap_out = 0;
  };

  template <typename T>
  static int grow(T*& p, size_t& cap, size_t n) {
    if (n <= cap) return MLB_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max(n, cap * 2);
    if (cudaMalloc((void**)&p, want * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      return MLB_ERR_OUT_OF_MEMORY;
    }
    cap = want;
    return MLB_OK;
  }

  // Runs a batch of small requests in one launch; sets each one's result
  // (the caller publishes it as the status, with the completion time).
  void run_small(std::vector<Request*>& batch, SmallBufs& B) {
    const int dtype = batch[0]->dtype;
    std::vector<mlb::SmallItem> items;
    std::vector<mlb_op_t> ops;
    std::vector<double> uni;
    std::vector<Request*> live;
    uint32_t nmax = 1;
    for (Request* r : batch) {
      std::vector<mlb_op_t> o;
      const int rc = mlb::prepare_ops(r->gates.data(), r->gates.size(), r->n, o);
      if (rc) {
        r->result = rc;
        continue;
      }
      mlb::SmallItem it{};
      it.ops_off = ops.size();
      it.num_ops = (uint32_t)o.size();
      it.n = r->n;
      it.shots = r->shots;
      it.uni_off = uni.size();
      it.out_off = uni.size();
      ops.insert(ops.end(), o.begin(), o.end());
      uint64_t seed = r->seed ? r->seed : ((uint64_t)std::time(nullptr) ^ 0x9e3779b97f4a7c15ULL);
      for (uint32_t k = 0; k < r->shots; k++) uni.push_back((double)(xorshift64(seed) >> 11) / (double)(1ULL << 53));
      items.push_back(it);
      live.push_back(r);
      nmax = std::max(nmax, r->n);
    }
    if (live.empty()) return;
    int rc = MLB_OK;
    if (!B.stream && cudaStreamCreateWithPriority(&B.stream, cudaStreamNonBlocking, prio_greatest) != cudaSuccess)
      rc = MLB_ERR_DRIVER;
    if (!rc) rc = grow(B.items, B.cap_items, items.size());
    if (!rc) rc = grow(B.ops, B.cap_ops, std::max<size_t>(1, ops.size()));
    if (!rc) rc = grow(B.uni, B.cap_uni, std::max<size_t>(1, uni.size()));
    if (!rc) rc = grow(B.out, B.cap_out, std::max<size_t>(1, uni.size()));
    std::vector<unsigned long long> out(uni.size());
    if (!rc) {
      cudaMemcpyAsync(B.items, items.data(), items.size() * sizeof(mlb::SmallItem), cudaMemcpyHostToDevice, B.stream);
      if (!ops.empty())
        cudaMemcpyAsync(B.ops, ops.data(), ops.size() * sizeof(mlb_op_t), cudaMemcpyHostToDevice, B.stream);
      if (!uni.empty())
        cudaMemcpyAsync(B.uni, uni.data(), uni.size() * sizeof(double), cudaMemcpyHostToDevice, B.stream);
      int sms = 148;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
      rc = mlb::launch_small_circuits(dtype, B.items, (int)items.size(), B.ops, B.uni, B.out, nmax, sms, B.stream);
      if (!rc && !uni.empty())
        cudaMemcpyAsync(out.data(), B.out, out.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                        B.stream);
      if (!rc && cudaStreamSynchronize(B.stream) != cudaSuccess) rc = MLB_ERR_DRIVER;
    }
    for (size_t i = 0; i < live.size(); i++) {
      Request* r = live[i];
      if (!rc) r->outcomes.assign(out.begin() + items[i].out_off, out.begin() + items[i].out_off + r->shots);
      r->result = rc;
    }
  }

  void worker() {
    cudaSetDevice(device);
    SmallBufs sbufs;
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      mlb_state_t* state = nullptr;
      std::vector<mlb_state_t*> evict;
      Request* r = nullptr;
      while (!stopping && !(r = pick(&state, &evict))) cv_work.wait(lk);
      if (!r) {  // stopping
        lk.unlock();
        for (void* p : {(void*)sbufs.items, (void*)sbufs.ops, (void*)sbufs.uni, (void*)sbufs.out})
          if (p) cudaFree(p);
        if (sbufs.stream) cudaStreamDestroy(sbufs.stream);
        return;
      }
      if (is_small(r)) {
        std::vector<Request*> batch{r};
        for (auto it = pending.begin(); it != pending.end() && batch.size() < kMaxSmallBatch;) {
          if (is_small(*it) && (*it)->dtype == r->dtype) {
            batch.push_back(*it);
            it = pending.erase(it);
          } else {
            ++it;
          }
        }
        const double ta = now();
        for (Request* q : batch) {
          q->status = 2;
          q->t_admit = ta;
        }
        running += (int)batch.size();
        st.peak_running = std::max<uint64_t>(st.peak_running, (uint64_t)running);
        st.small_batches++;
        st.small_requests += batch.size();
        lk.unlock();
        run_small(batch, sbufs);
        lk.lock();
        running -= (int)batch.size();
        // outcome and completion time become visible together, under mu: a
        // waiter may take (and delete) a request as soon as its status is final
        const double td = now();
        for (Request* q : batch) {
          q->status = q->result;
          q->t_done = td;
          if (q->status) st.failed++;
          st.completed++;
        }
        cv_done.notify_all();
        cv_work.notify_all();
        continue;
      }
      r->status = 2;
      r->t_admit = now();
      running++;
      st.peak_running = std::max<uint64_t>(st.peak_running, (uint64_t)running);
      st.peak_reserved_bytes = std::max<uint64_t>(st.peak_reserved_bytes, reserved);
      lk.unlock();

      for (mlb_state_t* e : evict) free_state(e);
      int rc = MLB_OK;
      if (!state) rc = new_state(r->n, r->dtype, &state);
      if (!rc) rc = mlb_state_reset(state);
      if (!rc) rc = mlb_run_gates(state, r->gates.data(), r->gates.size());
      if (!rc && r->shots) {
        uint64_t seed = r->seed ? r->seed : ((uint64_t)std::time(nullptr) ^ 0x9e3779b97f4a7c15ULL);
        std::vector<double> u(r->shots);
        for (auto& x : u) x = (double)(xorshift64(seed) >> 11) / (double)(1ULL << 53);
        r->outcomes.resize(r->shots);
        rc = mlb_sample(state, MLB_SAMPLE_CUM_GT, u.data(), u.size(), r->outcomes.data());
      } else if (!rc) {
        rc = mlb_synchronize(state);
      }
      uint64_t hit = 0;
      if (!rc) {
        mlb_flush_stats_t fs{};
        if (mlb_last_flush_stats(state, &fs) == MLB_OK) hit = fs.plan_cache_hit;
      }
      if (rc && state) {  // do not pool a state in an unknown condition
        free_state(state);
        state = nullptr;
      }

      lk.lock();
      running--;
      if (state) {
        idle[std::make_pair(r->n, r->dtype)].push_back(state);
      } else {
        reserved -= r->bytes;
      }
      r->status = rc;
      r->t_done = now();
      if (rc) st.failed++;
      st.completed++;
      st.plan_cache_hits += hit;
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }
};

extern "C" {

int mlb_server_create(int device, size_t hbm_budget_bytes, int num_workers, mlb_server_t** out) {
  if (!out) return mlb::record_error(MLB_ERR_INVALID_ARG, "null out");
  *out = nullptr;
  int cnt = 0;
  if (mlb_device_count(&cnt) != MLB_OK || device < 0 || device >= cnt)
    return mlb::record_error(MLB_ERR_NO_DEVICE, "no such device");
  if (num_workers < 1 || num_workers > 256)
    return mlb::record_error(MLB_ERR_INVALID_ARG, "num_workers must be 1..256");
  if (hbm_budget_bytes == 0) {
    size_t fr = 0, tot = 0;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaError_t e = cudaMemGetInfo(&fr, &tot);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return mlb::record_error(MLB_ERR_DRIVER, "cudaMemGetInfo failed");
    hbm_budget_bytes = fr / 10 * 8;  // 80 % of what is free now
  }
  auto* s = new (std::nothrow) mlb_server();
  if (!s) return mlb::record_error(MLB_ERR_OUT_OF_MEMORY, "host allocation");
  s->device = device;
  s->budget = hbm_budget_bytes;
  s->num_workers = num_workers;
  s->t0 = Clock::now();
  s->st.budget_bytes = hbm_budget_bytes;
  {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaDeviceGetStreamPriorityRange(&s->prio_least, &s->prio_greatest);
    cudaSetDevice(prev);
  }
  try {
    for (int i = 0; i < num_workers; i++) s->threads.emplace_back([s] { s->worker(); });
  } catch (...) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->threads) t.join();
    delete s;
    return mlb::record_error(MLB_ERR_OUT_OF_MEMORY, "thread creation failed");
  }
  *out = s;
  return MLB_OK;
}

int mlb_server_submit(mlb_server_t* s, const mlb_request_t* req, uint64_t* ticket) {
  if (!s || !req || !ticket || (req->num_gates && !req->gates))
    return mlb::record_error(MLB_ERR_INVALID_ARG, "null argument");
  if (req->dtype != MLB_C128 && req->dtype != MLB_C64)
    return mlb::record_error(MLB_ERR_INVALID_ARG, "dtype must be MLB_C128 or MLB_C64");
  const uint32_t maxq = req->dtype == MLB_C128 ? 33 : 34;
  if (req->num_qubits < 1 || req->num_qubits > maxq)
    return mlb::record_error(MLB_ERR_NUM_QUBITS, "num_qubits outside 1..33 (c128) / 1..34 (c64)");
  auto* r = new (std::nothrow) Request();
  if (!r) return mlb::record_error(MLB_ERR_OUT_OF_MEMORY, "host allocation");
  r->n = req->num_qubits;
  r->dtype = req->dtype;
  r->shots = req->num_shots;
  r->seed = req->rng_seed;
  r->bytes = state_bytes(r->n, r->dtype);
  try {
    r->gates.assign(req->gates, req->gates + req->num_gates);
  } catch (...) {
    delete r;
    return mlb::record_error(MLB_ERR_OUT_OF_MEMORY, "host allocation");
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (r->bytes > s->budget) {
    delete r;
    return mlb::record_error(MLB_ERR_OUT_OF_MEMORY, "request larger than the server's HBM budget");
  }
  if (s->stopping) {
    delete r;
    return mlb::record_error(MLB_ERR_BUSY, "server is shutting down");
  }
  r->ticket = s->next_ticket++;
  r->t_submit = s->now();
  s->pending.push_back(r);
  s->by_ticket[r->ticket] = r;
  s->st.submitted++;
  *ticket = r->ticket;
  s->cv_work.notify_one();
  return MLB_OK;
}

int mlb_server_wait(mlb_server_t* s, uint64_t ticket, int timeout_ms, uint64_t* outcomes,
                    size_t capacity, mlb_request_info_t* info) {
  if (!s) return mlb::record_error(MLB_ERR_INVALID_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->by_ticket.find(ticket);
  if (it == s->by_ticket.end()) return mlb::record_error(MLB_ERR_INVALID_ARG, "unknown ticket");
  Request* r = it->second;
  auto done = [&] { return r->status != 1 && r->status != 2; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, done);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
    return MLB_ERR_TIMEOUT;
  }
  if (outcomes && r->status == MLB_OK) {
    if (capacity < r->outcomes.size())
      return mlb::record_error(MLB_ERR_INVALID_ARG, "outcome buffer smaller than num_shots");
    if (!r->outcomes.empty()) std::memcpy(outcomes, r->outcomes.data(), r->outcomes.size() * sizeof(uint64_t));
  }
  if (info) {
    info->status = r->status;
    info->num_qubits = r->n;
    info->dtype = r->dtype;
    info->num_shots = r->shots;
    info->submit_s = r->t_submit;
    info->admit_s = r->t_admit;
    info->done_s = r->t_done;
  }
  const int rc = r->status;
  s->by_ticket.erase(it);
  delete r;
  return rc;
}

int mlb_server_get_stats(mlb_server_t* s, mlb_server_stats_t* out) {
  if (!s || !out) return mlb::record_error(MLB_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->pending = s->pending.size();
  out->running = (uint64_t)s->running;
  out->reserved_bytes = s->reserved;
  return MLB_OK;
}

void mlb_server_destroy(mlb_server_t* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    for (Request* r : s->pending) {  // never admitted: cancelled
      r->status = MLB_ERR_BUSY;
      r->t_done = s->now();
    }
    s->pending.clear();
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  for (auto& t : s->threads) t.join();  // running requests finish first
  for (auto& kv : s->idle)
    for (mlb_state_t* st : kv.second) s->free_state(st);
  for (auto& kv : s->by_ticket) delete kv.second;
  delete s;
}

}  // extern "C"
