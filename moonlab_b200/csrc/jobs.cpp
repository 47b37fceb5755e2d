// jobs.cpp -- scheduler jobs on the engine: the moonlab_job_to_json reader,
// the "simulator"-backend semantics on the GPU (mlb_job_run) and the "b200"
// backend plug-in for the reference's registry.
//
// Reference: src/distributed/scheduler.{h,c} (job, registry at :283-305,
// simulator_backend_execute :194-239, run_worker_slice :152-191,
// moonlab_job_to_json :492-537) and src/applications/moonlab_qgtl_backend.c
// (xorshift64 shot uniforms :158-167, :226-240).
//
// The reference runs the circuit once per worker and clones the state once
// per shot; every worker computes the same output state, and each shot is
// measurement_all_qubits(u) on it.  Here the circuit runs once on the GPU and
// all shots are sampled from that state with the same uniforms, which gives
// the same outcomes.
#include <dlfcn.h>

#include <atomic>
#include <cerrno>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <mutex>
#include <string>
#include <vector>

#include "moonlab_b200.h"
#include "moonlab_b200_dropin.h"
#include "mlb_internal.h"

namespace {

// ---- scheduler status codes (scheduler.h:36-42) ---------------------------
constexpr int kSchedOk = 0, kSchedBadArg = -501, kSchedOom = -502, kSchedInternal = -503,
              kSchedBackendNotFound = -506;

// moonlab_job_results_t (scheduler.h:51-57).
struct JobResults {
  int num_qubits;
  int total_shots;
  uint64_t* outcomes;
  int num_workers_used;
  double* worker_seconds;
};

// moonlab_backend_t (scheduler.h:244-249).
struct Backend {
  const char* name;
  int (*execute)(const void*, void*, void*);
  void* ctx;
  const char* description;
};

using RegisterFn = int (*)(const Backend*);
using ToJsonFn = int (*)(const void*, char*, size_t);

// ---- the job text -----------------------------------------------------------
// A small reader for the JSON that moonlab_job_to_json writes.  It accepts any
// well-formed JSON of that shape (key order free, unknown keys skipped).
struct Reader {
  const char* p;
  bool ok = true;

  void ws() {
    while (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t') p++;
  }
  bool eat(char c) {
    ws();
    if (*p != c) return false;
    p++;
    return true;
  }
  bool string(std::string& out) {
    ws();
    if (*p != '"') return false;
    p++;
    out.clear();
    while (*p && *p != '"') {
      if (*p == '\\') {
        p++;
        if (!*p) return false;
      }
      out.push_back(*p++);
    }
    if (*p != '"') return false;
    p++;
    return true;
  }
  bool number(double& v, long long& iv, bool& is_int) {
    ws();
    const char* s = p;
    if (*p == '-' || *p == '+') p++;
    bool any = false;
    while ((*p >= '0' && *p <= '9') || *p == '.' || *p == 'e' || *p == 'E' || *p == '-' || *p == '+') {
      any = true;
      p++;
    }
    if (!any) return false;
    std::string tok(s, p);
    is_int = tok.find_first_of(".eE") == std::string::npos;
    errno = 0;
    char* end = nullptr;
    if (is_int) {
      iv = std::strtoll(tok.c_str(), &end, 10);
      v = (double)iv;
    } else {
      v = std::strtod(tok.c_str(), &end);  // %.17g text: exact round trip
    }
    return end && *end == '\0' && errno == 0;
  }
  bool skip_value(int depth = 0) {
    if (depth > 64) return false;
    ws();
    if (*p == '"') {
      std::string s;
      return string(s);
    }
    if (*p == '{' || *p == '[') {
      const char close = *p == '{' ? '}' : ']';
      const bool obj = *p == '{';
      p++;
      if (eat(close)) return true;
      for (;;) {
        if (obj) {
          std::string k;
          if (!string(k) || !eat(':')) return false;
        }
        if (!skip_value(depth + 1)) return false;
        if (eat(',')) continue;
        return eat(close);
      }
    }
    for (const char* lit : {"true", "false", "null"}) {
      const size_t L = std::strlen(lit);
      if (std::strncmp(p, lit, L) == 0) {
        p += L;
        return true;
      }
    }
    double v;
    long long iv;
    bool is_int;
    return number(v, iv, is_int);
  }
  bool integer(long long& iv) {
    double v;
    bool is_int;
    return number(v, iv, is_int) && is_int;
  }
};

bool parse_gate(Reader& r, mlb_gate_t& g) {
  if (!r.eat('{')) return false;
  g = mlb_gate_t{0, -1, -1, 0, 0.0};
  bool have_type = false, have_target = false;
  if (r.eat('}')) return false;
  for (;;) {
    std::string key;
    if (!r.string(key) || !r.eat(':')) return false;
    long long iv;
    if (key == "type" || key == "target" || key == "control") {
      if (!r.integer(iv) || iv < INT32_MIN || iv > INT32_MAX) return false;
      if (key == "type") g.type = (int32_t)iv, have_type = true;
      else if (key == "target") g.target = (int32_t)iv, have_target = true;
      else g.control = (int32_t)iv;
    } else if (key == "theta") {
      double v;
      bool is_int;
      if (!r.number(v, iv, is_int)) return false;
      g.theta = v;
    } else if (!r.skip_value()) {
      return false;
    }
    if (r.eat(',')) continue;
    if (!r.eat('}')) return false;
    return have_type && have_target;
  }
}

int parse_job(const char* json, mlb_job_desc_t& d, std::vector<mlb_gate_t>& gates) {
  Reader r{json};
  d = mlb_job_desc_t{0, 0, 1, 0, 0};
  bool have_n = false, have_gates = false;
  gates.clear();
  if (!r.eat('{')) return MLB_ERR_INVALID_ARG;
  if (!r.eat('}')) {
    for (;;) {
      std::string key;
      if (!r.string(key) || !r.eat(':')) return MLB_ERR_INVALID_ARG;
      long long iv;
      if (key == "num_qubits" || key == "num_shots" || key == "num_workers") {
        if (!r.integer(iv) || iv < INT32_MIN || iv > INT32_MAX) return MLB_ERR_INVALID_ARG;
        if (key == "num_qubits") d.num_qubits = (int32_t)iv, have_n = true;
        else if (key == "num_shots") d.num_shots = (int32_t)iv;
        else d.num_workers = (int32_t)iv;
      } else if (key == "rng_seed") {
        r.ws();
        if (*r.p == '"') {  // "0x%016llx"
          std::string s;
          if (!r.string(s)) return MLB_ERR_INVALID_ARG;
          errno = 0;
          char* end = nullptr;
          d.rng_seed = std::strtoull(s.c_str(), &end, 16);
          if (s.empty() || !end || *end != '\0' || errno) return MLB_ERR_INVALID_ARG;
        } else {
          if (!r.integer(iv) || iv < 0) return MLB_ERR_INVALID_ARG;
          d.rng_seed = (uint64_t)iv;
        }
      } else if (key == "gates") {
        if (!r.eat('[')) return MLB_ERR_INVALID_ARG;
        have_gates = true;
        if (!r.eat(']')) {
          for (;;) {
            mlb_gate_t g;
            if (!parse_gate(r, g)) return MLB_ERR_INVALID_ARG;
            gates.push_back(g);
            if (r.eat(',')) continue;
            if (!r.eat(']')) return MLB_ERR_INVALID_ARG;
            break;
          }
        }
      } else if (!r.skip_value()) {
        return MLB_ERR_INVALID_ARG;
      }
      if (r.eat(',')) continue;
      if (!r.eat('}')) return MLB_ERR_INVALID_ARG;
      break;
    }
  }
  r.ws();
  if (*r.p != '\0' || !have_n || !have_gates) return MLB_ERR_INVALID_ARG;
  return MLB_OK;
}

// ---- seeds and uniforms ------------------------------------------------------
uint64_t splitmix64_mix(uint64_t x) {  // scheduler.c:143-148
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d49bb133111ebbULL;
  return x ^ (x >> 31);
}
uint64_t xorshift64(uint64_t& s) {  // moonlab_qgtl_backend.c:159-167
  uint64_t x = s;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  s = x;
  return x;
}
constexpr uint64_t kGolden = 0x9e3779b97f4a7c15ULL;

// ---- one cached device state (jobs of the same width reuse it) --------------
std::mutex g_job_mu;
mlb_state_t* g_state = nullptr;
uint32_t g_state_n = 0;
int g_state_dev = -1;

void release_locked() {
  if (g_state) mlb_state_free(g_state);
  g_state = nullptr;
  g_state_n = 0;
  g_state_dev = -1;
}

std::atomic<ToJsonFn> g_to_json{nullptr};

}  // namespace

extern "C" {

int mlb_job_parse_json(const char* json, mlb_job_desc_t* desc, mlb_gate_t* gates, size_t capacity,
                       size_t* num_gates) {
  if (!json || !desc || !num_gates) return mlb::record_error(MLB_ERR_INVALID_ARG, "null argument");
  std::vector<mlb_gate_t> g;
  mlb_job_desc_t d;
  if (parse_job(json, d, g) != MLB_OK)
    return mlb::record_error(MLB_ERR_INVALID_ARG, "job text is not moonlab_job_to_json JSON");
  *desc = d;
  *num_gates = g.size();
  if (!gates) return MLB_OK;
  if (capacity < g.size()) return mlb::record_error(MLB_ERR_INVALID_ARG, "gate buffer too small");
  if (!g.empty()) std::memcpy(gates, g.data(), g.size() * sizeof(mlb_gate_t));
  return MLB_OK;
}

int mlb_job_run(const mlb_job_desc_t* desc, const mlb_gate_t* gates, size_t num_gates, int device,
                uint64_t* outcomes, int* workers_used, double* seconds) {
  if (!desc || !outcomes || (num_gates && !gates))
    return mlb::record_error(MLB_ERR_INVALID_ARG, "null argument");
  if (desc->num_shots <= 0) return mlb::record_error(MLB_ERR_INVALID_ARG, "num_shots must be > 0");
  if (desc->num_qubits < 1) return mlb::record_error(MLB_ERR_NUM_QUBITS, "num_qubits must be >= 1");
  const auto t0 = std::chrono::steady_clock::now();
  const int total = desc->num_shots;
  int workers = desc->num_workers;
  if (workers > total) workers = total;
  if (workers < 1) workers = 1;

  // Uniforms of every worker slice, in outcome order.
  std::vector<double> u((size_t)total);
  for (int w = 0; w < workers; w++) {
    const int start = (int)((long long)w * total / workers);
    const int end = (int)((long long)(w + 1) * total / workers);
    uint64_t seed = desc->rng_seed
                        ? splitmix64_mix(desc->rng_seed ^ ((uint64_t)w << 32))
                        : ((uint64_t)std::time(nullptr) ^ ((uint64_t)w << 32) ^ kGolden);
    if (seed == 0) seed = (uint64_t)std::time(nullptr) ^ kGolden;
    for (int s = start; s < end; s++) u[(size_t)s] = (double)(xorshift64(seed) >> 11) / (double)(1ULL << 53);
  }

  std::lock_guard<std::mutex> lk(g_job_mu);
  const uint32_t n = (uint32_t)desc->num_qubits;
  if (!g_state || g_state_n != n || g_state_dev != device) {
    release_locked();
    int rc = mlb_state_create(n, MLB_C128, device, &g_state);
    if (rc) {
      g_state = nullptr;
      return rc;
    }
    g_state_n = n;
    g_state_dev = device;
  }
  int rc = mlb_state_reset(g_state);
  if (!rc) rc = mlb_run_gates(g_state, gates, num_gates);
  if (!rc) rc = mlb_sample(g_state, MLB_SAMPLE_CUM_GT, u.data(), u.size(), outcomes);
  if (rc) {
    // keep the error text of the failing call; drop the state (it may be
    // half-updated) so the next job starts clean
    std::string msg = mlb_last_error();
    release_locked();
    return mlb::record_error(rc, msg.c_str());
  }
  if (workers_used) *workers_used = workers;
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return MLB_OK;
}

int moonlab_b200_backend_execute(const void* job, void* results, void* ctx) {
  if (!job || !results) return kSchedBadArg;
  ToJsonFn to_json = g_to_json.load();
  if (!to_json) to_json = (ToJsonFn)dlsym(RTLD_DEFAULT, "moonlab_job_to_json");
  if (!to_json) return kSchedInternal;
  const int len = to_json(job, nullptr, 0);
  if (len <= 0) return kSchedInternal;
  std::string text((size_t)len + 1, '\0');
  if (to_json(job, &text[0], text.size()) != len) return kSchedInternal;
  mlb_job_desc_t d;
  std::vector<mlb_gate_t> gates;
  if (parse_job(text.c_str(), d, gates) != MLB_OK) return kSchedInternal;
  if (d.num_shots <= 0) return kSchedBadArg;

  JobResults* out = (JobResults*)results;
  int workers = d.num_workers > d.num_shots ? d.num_shots : (d.num_workers < 1 ? 1 : d.num_workers);
  out->num_qubits = d.num_qubits;
  out->total_shots = d.num_shots;
  out->num_workers_used = workers;
  out->outcomes = (uint64_t*)std::malloc((size_t)d.num_shots * sizeof(uint64_t));
  out->worker_seconds = (double*)std::calloc((size_t)workers, sizeof(double));
  if (!out->outcomes || !out->worker_seconds) return kSchedOom;
  const int device = ctx ? *(const int*)ctx : 0;
  double secs = 0.0;
  const int rc = mlb_job_run(&d, gates.data(), gates.size(), device, out->outcomes, &workers, &secs);
  if (rc == MLB_ERR_OUT_OF_MEMORY) return kSchedOom;
  if (rc) return kSchedInternal;
  // One GPU run serves every slice; report its time split by slice size.
  for (int w = 0; w < workers; w++) {
    const long long a = (long long)w * d.num_shots / workers, b = (long long)(w + 1) * d.num_shots / workers;
    out->worker_seconds[w] = secs * (double)(b - a) / (double)d.num_shots;
  }
  return kSchedOk;
}

int moonlab_b200_register_backend_with(void* register_fn, void* job_to_json_fn) {
  if (!register_fn || !job_to_json_fn) return kSchedBadArg;
  g_to_json.store((ToJsonFn)job_to_json_fn);
  static const Backend be = {"b200", &moonlab_b200_backend_execute, nullptr,
                             "B200 (sm_100a) state-vector engine, complex128; outcomes identical to "
                             "\"simulator\" for a non-zero seed."};
  return ((RegisterFn)register_fn)(&be);
}

int moonlab_b200_register_backend(void) {
  void* reg = dlsym(RTLD_DEFAULT, "moonlab_register_backend");
  if (!reg) return kSchedBackendNotFound;
  // moonlab_job_to_json from the same library as the registry
  void* to_json = nullptr;
  Dl_info info;
  if (dladdr(reg, &info) && info.dli_fname) {
    void* h = dlopen(info.dli_fname, RTLD_LAZY | RTLD_NOLOAD);
    if (h) {
      to_json = dlsym(h, "moonlab_job_to_json");
      dlclose(h);
    }
  }
  if (!to_json) to_json = dlsym(RTLD_DEFAULT, "moonlab_job_to_json");
  if (!to_json) return kSchedBackendNotFound;
  return moonlab_b200_register_backend_with(reg, to_json);
}

void moonlab_b200_release_backend_state(void) {
  std::lock_guard<std::mutex> lk(g_job_mu);
  release_locked();
}

}  // extern "C"
