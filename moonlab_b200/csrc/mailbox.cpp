// mailbox.cpp -- host side of the persistent small-circuit loop
// (kernels_mailbox.cu): requests are posted into a device-memory ring and
// served by one long-running launch, so a small request costs two copies
// and a flag instead of a kernel launch and a stream synchronisation.
//
// Posting (mlb_mailbox_submit, one producer at a time under a mutex): the
// request's ops and uniforms go into its slot's pinned staging buffers, then
// three copies on the mailbox's copy stream -- ops, uniforms, descriptor --
// and a fourth that writes the new `tail`; stream order puts the data in
// device memory before the count that publishes it.  The slot's done word
// (mapped host memory) is cleared first; the kernel sets it to seq + 1 after
// the outcomes, which it writes straight into mapped host memory.
//
// The kernel's blocks exit after idle_ms without a request (a bounded wait;
// the launch then ends with MLB_ERR_TIMEOUT, counted in the stats) or when
// the stop word is set (mlb_mailbox_free).  Submit relaunches the loop when
// it has ended, and so does a waiter that finds its request still pending on
// an ended launch, so a posted request is always served.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <ctime>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "moonlab_b200.h"
#include "mlb_internal.h"

namespace {

uint64_t mb_xorshift64(uint64_t& s) {  // moonlab_qgtl_backend.c:159-167
  uint64_t x = s;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  s = x;
  return x;
}

constexpr uint64_t kFree = ~0ull;

}  // namespace

struct mlb_mailbox {
  int dtype = MLB_C128, device = 0, ctas = 8;
  uint32_t slots = 64, max_ops = 2048, max_shots = 4096, nmax = 12;
  uint64_t idle_ns = 1000000000ull;
  cudaStream_t kstream = nullptr, cstream = nullptr;
  // device memory
  mlb::MailboxItem* d_items = nullptr;
  mlb_op_t* d_ops = nullptr;
  double* d_uni = nullptr;
  uint64_t* d_ctl = nullptr;  // [0] head, [1] tail, [2] stop (low word), [3] exited (low word), [4] end status
  // pinned host memory: staging per slot, the tail value per slot, the stop word
  mlb::MailboxItem* h_items = nullptr;
  mlb_op_t* h_ops = nullptr;
  double* h_uni = nullptr;
  uint64_t* h_tail = nullptr;
  uint32_t* h_stop = nullptr;
  // mapped host memory written by the kernel
  unsigned long long* h_out = nullptr;
  volatile uint64_t* h_done = nullptr;
  std::mutex mu;
  uint64_t next_seq = 0;
  std::vector<uint64_t> slot_seq;
  std::vector<uint32_t> slot_shots;
  bool launched = false;
  mlb_mailbox_stats_t stats{};

  mlb::MailboxDev dev() const {
    mlb::MailboxDev m{};
    m.items = d_items;
    m.ops = d_ops;
    m.uniforms = d_uni;
    unsigned long long* out_dev = nullptr;
    uint64_t* done_dev = nullptr;
    cudaHostGetDevicePointer((void**)&out_dev, h_out, 0);
    cudaHostGetDevicePointer((void**)&done_dev, (void*)h_done, 0);
    m.outcomes = out_dev;
    m.done = done_dev;
    m.head = d_ctl;
    m.tail = d_ctl + 1;
    m.stop = reinterpret_cast<const uint32_t*>(d_ctl + 2);
    m.exited = reinterpret_cast<uint32_t*>(d_ctl + 3);
    m.end_status = reinterpret_cast<int*>(d_ctl + 4);
    m.idle_ns = idle_ns;
    m.slots = slots;
    m.max_ops = max_ops;
    m.max_shots = max_shots;
    m.nmax = nmax;
    return m;
  }

  // The loop's launch has ended (or never ran): record how, and start it.
  // Called with mu held.
  int ensure_running() {
    if (launched) {
      const cudaError_t q = cudaStreamQuery(kstream);
      if (q == cudaErrorNotReady) return MLB_OK;
      if (q != cudaSuccess) return MLB_ERR_DRIVER;
      int end = MLB_OK;
      if (cudaMemcpy(&end, d_ctl + 4, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return MLB_ERR_DRIVER;
      if (end == MLB_ERR_TIMEOUT) stats.idle_exits++;
      launched = false;
    }
    if (cudaMemsetAsync(d_ctl + 3, 0, 2 * sizeof(uint64_t), kstream) != cudaSuccess) return MLB_ERR_DRIVER;
    const int rc = mlb::launch_mailbox(dtype, dev(), ctas, kstream);
    if (rc) return rc;
    launched = true;
    stats.launches++;
    return MLB_OK;
  }

  void release() {
    if (kstream) cudaStreamSynchronize(kstream);
    if (cstream) cudaStreamSynchronize(cstream);
    cudaFree(d_items);
    cudaFree(d_ops);
    cudaFree(d_uni);
    cudaFree(d_ctl);
    cudaFreeHost(h_items);
    cudaFreeHost(h_ops);
    cudaFreeHost(h_uni);
    cudaFreeHost(h_tail);
    cudaFreeHost(h_stop);
    cudaFreeHost(h_out);
    cudaFreeHost((void*)h_done);
    if (kstream) cudaStreamDestroy(kstream);
    if (cstream) cudaStreamDestroy(cstream);
  }
};

extern "C" {

int mlb_mailbox_create(const mlb_mailbox_config_t* cfg, mlb_mailbox_t** out) {
  if (!out) return mlb::record_error(MLB_ERR_INVALID_ARG, "mailbox: null output");
  *out = nullptr;
  auto* mb = new mlb_mailbox();
  if (cfg) {
    if (cfg->dtype != MLB_C128 && cfg->dtype != MLB_C64) {
      delete mb;
      return mlb::record_error(MLB_ERR_INVALID_ARG, "mailbox: dtype must be MLB_C128 or MLB_C64");
    }
    mb->dtype = cfg->dtype;
    mb->device = cfg->device;
    if (cfg->ctas > 0) mb->ctas = cfg->ctas;
    if (cfg->slots > 0) mb->slots = cfg->slots;
    if (cfg->max_ops > 0) mb->max_ops = cfg->max_ops;
    if (cfg->max_shots > 0) mb->max_shots = cfg->max_shots;
    if (cfg->idle_ms > 0) mb->idle_ns = (uint64_t)(cfg->idle_ms * 1e6);
  }
  mb->nmax = (uint32_t)mlb::small_max_qubits(mb->dtype);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || mb->device < 0 || mb->device >= ndev) {
    cudaGetLastError();
    delete mb;
    return mlb::record_error(MLB_ERR_NO_DEVICE, "mailbox: no such CUDA device");
  }
  int sms = 0;
  cudaSetDevice(mb->device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, mb->device);
  if (mb->ctas > sms) mb->ctas = sms;
  const size_t S = mb->slots;
  bool ok = cudaStreamCreateWithFlags(&mb->kstream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&mb->cstream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc((void**)&mb->d_items, S * sizeof(mlb::MailboxItem)) == cudaSuccess &&
            cudaMalloc((void**)&mb->d_ops, S * mb->max_ops * sizeof(mlb_op_t)) == cudaSuccess &&
            cudaMalloc((void**)&mb->d_uni, S * mb->max_shots * sizeof(double)) == cudaSuccess &&
            cudaMalloc((void**)&mb->d_ctl, 8 * sizeof(uint64_t)) == cudaSuccess &&
            cudaHostAlloc((void**)&mb->h_items, S * sizeof(mlb::MailboxItem), cudaHostAllocDefault) == cudaSuccess &&
            cudaHostAlloc((void**)&mb->h_ops, S * mb->max_ops * sizeof(mlb_op_t), cudaHostAllocDefault) == cudaSuccess &&
            cudaHostAlloc((void**)&mb->h_uni, S * mb->max_shots * sizeof(double), cudaHostAllocDefault) == cudaSuccess &&
            cudaHostAlloc((void**)&mb->h_tail, S * sizeof(uint64_t), cudaHostAllocDefault) == cudaSuccess &&
            cudaHostAlloc((void**)&mb->h_stop, sizeof(uint32_t), cudaHostAllocDefault) == cudaSuccess &&
            cudaHostAlloc((void**)&mb->h_out, S * mb->max_shots * sizeof(unsigned long long), cudaHostAllocMapped) ==
                cudaSuccess &&
            cudaHostAlloc((void**)&mb->h_done, S * sizeof(uint64_t), cudaHostAllocMapped) == cudaSuccess &&
            cudaMemset(mb->d_ctl, 0, 8 * sizeof(uint64_t)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    mb->release();
    delete mb;
    return mlb::record_error(MLB_ERR_OUT_OF_MEMORY, "mailbox: allocation failed");
  }
  for (size_t i = 0; i < S; i++) mb->h_done[i] = 0;
  mb->slot_seq.assign(S, kFree);
  mb->slot_shots.assign(S, 0);
  *out = mb;
  return MLB_OK;
}

int mlb_mailbox_submit(mlb_mailbox_t* mb, const mlb_request_t* req, uint64_t* ticket) {
  if (!mb || !req || !ticket) return mlb::record_error(MLB_ERR_INVALID_ARG, "mailbox: null argument");
  if (req->dtype != mb->dtype) return mlb::record_error(MLB_ERR_INVALID_ARG, "mailbox: request dtype differs");
  if (req->num_qubits < 1 || req->num_qubits > mb->nmax)
    return mlb::record_error(MLB_ERR_NUM_QUBITS, "mailbox: request larger than a block's shared memory");
  if (req->num_shots > mb->max_shots) return mlb::record_error(MLB_ERR_INVALID_ARG, "mailbox: too many shots");
  std::vector<mlb_op_t> ops;
  int rc = mlb::prepare_ops(req->gates, req->num_gates, req->num_qubits, ops);
  if (rc) return rc;
  if (ops.size() > mb->max_ops) return mlb::record_error(MLB_ERR_INVALID_ARG, "mailbox: too many ops for a slot");
  std::lock_guard<std::mutex> lk(mb->mu);
  cudaSetDevice(mb->device);
  const uint64_t seq = mb->next_seq;
  const uint32_t slot = (uint32_t)(seq % mb->slots);
  if (mb->slot_seq[slot] != kFree) return MLB_ERR_BUSY;  // ring full: wait for older tickets first
  // staging (the slot's own pinned buffers: free until its ticket is waited)
  mlb_op_t* hops = mb->h_ops + (size_t)slot * mb->max_ops;
  double* huni = mb->h_uni + (size_t)slot * mb->max_shots;
  if (!ops.empty()) std::memcpy(hops, ops.data(), ops.size() * sizeof(mlb_op_t));
  uint64_t seed = req->rng_seed ? req->rng_seed : ((uint64_t)std::time(nullptr) ^ 0x9e3779b97f4a7c15ULL);
  for (uint32_t k = 0; k < req->num_shots; k++) huni[k] = (double)(mb_xorshift64(seed) >> 11) / (double)(1ULL << 53);
  mlb::MailboxItem& it = mb->h_items[slot];
  it.num_ops = (uint32_t)ops.size();
  it.n = req->num_qubits;
  it.shots = req->num_shots;
  it.pad = 0;
  mb->h_done[slot] = 0;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  mb->h_tail[slot] = seq + 1;
  bool ok = true;
  if (!ops.empty())
    ok = ok && cudaMemcpyAsync(mb->d_ops + (size_t)slot * mb->max_ops, hops, ops.size() * sizeof(mlb_op_t),
                               cudaMemcpyHostToDevice, mb->cstream) == cudaSuccess;
  if (req->num_shots)
    ok = ok && cudaMemcpyAsync(mb->d_uni + (size_t)slot * mb->max_shots, huni, req->num_shots * sizeof(double),
                               cudaMemcpyHostToDevice, mb->cstream) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(mb->d_items + slot, &it, sizeof(it), cudaMemcpyHostToDevice, mb->cstream) == cudaSuccess;
  // publish: stream order puts this after the request's data
  ok = ok && cudaMemcpyAsync(mb->d_ctl + 1, mb->h_tail + slot, sizeof(uint64_t), cudaMemcpyHostToDevice,
                             mb->cstream) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    return mlb::record_error(MLB_ERR_DRIVER, "mailbox: posting copies failed");
  }
  mb->slot_seq[slot] = seq;
  mb->slot_shots[slot] = req->num_shots;
  mb->next_seq = seq + 1;
  mb->stats.submitted++;
  rc = mb->ensure_running();
  if (rc) return mlb::record_error(rc, "mailbox: launching the request loop failed");
  *ticket = seq;
  return MLB_OK;
}

int mlb_mailbox_wait(mlb_mailbox_t* mb, uint64_t ticket, int timeout_ms, uint64_t* outcomes, size_t capacity) {
  if (!mb) return mlb::record_error(MLB_ERR_INVALID_ARG, "mailbox: null mailbox");
  const uint32_t slot = (uint32_t)(ticket % mb->slots);
  uint32_t shots = 0;
  {
    std::lock_guard<std::mutex> lk(mb->mu);
    if (mb->slot_seq[slot] != ticket) return mlb::record_error(MLB_ERR_INVALID_ARG, "mailbox: unknown ticket");
    shots = mb->slot_shots[slot];
  }
  if (shots && (!outcomes || capacity < shots))
    return mlb::record_error(MLB_ERR_INVALID_ARG, "mailbox: outcome buffer smaller than num_shots");
  const auto t0 = std::chrono::steady_clock::now();
  for (int spins = 0;; spins++) {
    if (mb->h_done[slot] == ticket + 1) break;
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (timeout_ms >= 0 && ms > timeout_ms) return MLB_ERR_TIMEOUT;
    if (spins % 64 == 63) {  // still pending on an ended launch: start it again
      std::lock_guard<std::mutex> lk(mb->mu);
      cudaSetDevice(mb->device);
      const int rc = mb->ensure_running();
      if (rc) return mlb::record_error(rc, "mailbox: relaunching the request loop failed");
    }
    if (spins > 256) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  if (shots)
    for (uint32_t k = 0; k < shots; k++) outcomes[k] = mb->h_out[(size_t)slot * mb->max_shots + k];
  std::lock_guard<std::mutex> lk(mb->mu);
  mb->slot_seq[slot] = kFree;
  mb->stats.completed++;
  return MLB_OK;
}

int mlb_mailbox_get_stats(mlb_mailbox_t* mb, mlb_mailbox_stats_t* out) {
  if (!mb || !out) return mlb::record_error(MLB_ERR_INVALID_ARG, "mailbox: null argument");
  std::lock_guard<std::mutex> lk(mb->mu);
  cudaSetDevice(mb->device);
  if (mb->launched && cudaStreamQuery(mb->kstream) == cudaSuccess) {  // ended: count how
    int end = MLB_OK;
    if (cudaMemcpy(&end, mb->d_ctl + 4, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
        end == MLB_ERR_TIMEOUT)
      mb->stats.idle_exits++;
    mb->launched = false;
  }
  *out = mb->stats;
  out->running = mb->launched ? 1 : 0;
  return MLB_OK;
}

int mlb_mailbox_free(mlb_mailbox_t* mb) {
  if (!mb) return MLB_OK;
  int rc = MLB_OK;
  {
    std::lock_guard<std::mutex> lk(mb->mu);
    cudaSetDevice(mb->device);
    *mb->h_stop = 1;
    if (cudaMemcpyAsync(mb->d_ctl + 2, mb->h_stop, sizeof(uint32_t), cudaMemcpyHostToDevice, mb->cstream) !=
            cudaSuccess ||
        cudaStreamSynchronize(mb->cstream) != cudaSuccess || cudaStreamSynchronize(mb->kstream) != cudaSuccess)
      rc = MLB_ERR_DRIVER;
  }
  mb->release();
  delete mb;
  return rc;
}

}  // extern "C"
