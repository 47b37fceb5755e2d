// control.cpp -- the control server's request execution on the device loop.
//
// Reference: src/control/control_plane.h:8-33 (wire frames) and
// control_plane.c:415-424 (HEALTH), :598-632 (verb line and limits),
// :667-686 (deserialize, qubit cap), :688-770 (moonlab_qgtl_execute and the
// response frames); status codes control_plane.h:54-62; limits :264-292.
//
// The reference's server reads a verb line and a body from a socket and
// runs the circuit with moonlab_qgtl_execute on the host, one request at a
// time per connection thread.  Here the same frame goes to the engine:
// SHOTS requests into the continuous-batching server (many requests overlap
// on the GPU), CIRCUIT requests onto a complex128 state of their own.  The
// transport (sockets, TLS, AUTH/HMAC, rate limits, METRICS, admission
// hooks) stays the reference's: a handler gets the frame that follows an
// AUTH line, if any.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "moonlab_b200.h"
#include "mlb_internal.h"

namespace {

// control_plane.h:54-62
constexpr int kCtlBadArg = -401, kCtlProtocol = -404, kCtlRejected = -405;
// control_plane.c:264-279
constexpr long kMaxBodyBytes = 1L << 22;
constexpr long kMaxShots = 1L << 20;
constexpr uint32_t kDefaultMaxQubits = 30;  // the reference's ceiling (its default is 24)
constexpr uint32_t kMaxQubitsC128 = 33;     // a complex128 state on one device (128 GiB)
constexpr size_t kVerbCap = 96;             // the reference's verb-line buffer

}  // namespace

struct mlb_control {
  int device = 0;
  size_t hbm_budget = 0;
  int num_workers = 8;
  uint32_t max_qubits = kDefaultMaxQubits;
  bool fixed_seed = false;
  uint64_t seed = 0;
  std::mutex server_mu;        // creation of the batching server at the first SHOTS request
  std::mutex circuit_mu;       // CIRCUIT requests run one at a time (a state and 2^n probabilities each)
  mlb_server_t* server = nullptr;
};

namespace {

struct Frame {
  std::string head;
  std::vector<uint8_t> payload;
};

Frame err_frame(int code, const char* msg) {
  char b[128];
  std::snprintf(b, sizeof b, "ERR %d %s\n", code, msg);
  return Frame{b, {}};
}

int shots_request(mlb_control* c, uint32_t n, const std::vector<mlb_gate_t>& gates, long shots, Frame& out) {
  mlb_server_t* srv = nullptr;
  {
    std::lock_guard<std::mutex> lk(c->server_mu);
    if (!c->server && mlb_server_create(c->device, c->hbm_budget, c->num_workers, &c->server) != MLB_OK) {
      out = err_frame(kCtlRejected, "execute");
      return MLB_OK;
    }
    srv = c->server;
  }
  mlb_request_t rq{};
  rq.num_qubits = n;
  rq.dtype = MLB_C128;
  rq.gates = gates.data();
  rq.num_gates = gates.size();
  rq.num_shots = (uint32_t)shots;
  rq.rng_seed = c->fixed_seed ? c->seed : 0;  // 0: the clock, as the reference's server
  uint64_t ticket = 0;
  std::vector<uint64_t> outcomes((size_t)shots);
  if (mlb_server_submit(srv, &rq, &ticket) != MLB_OK ||
      mlb_server_wait(srv, ticket, -1, outcomes.data(), outcomes.size(), nullptr) != MLB_OK) {
    out = err_frame(kCtlRejected, "execute");
    return MLB_OK;
  }
  char b[64];
  std::snprintf(b, sizeof b, "SAMPLES %ld\n", shots);
  out.head = b;
  out.payload.resize(outcomes.size() * sizeof(uint64_t));
  std::memcpy(out.payload.data(), outcomes.data(), out.payload.size());
  return MLB_OK;
}

int circuit_request(mlb_control* c, uint32_t n, const std::vector<mlb_gate_t>& gates, Frame& out) {
  std::lock_guard<std::mutex> lk(c->circuit_mu);
  mlb_state_t* s = nullptr;
  const size_t dim = (size_t)1 << n;
  std::vector<uint8_t> probs;
  bool ok = mlb_state_create(n, MLB_C128, c->device, &s) == MLB_OK;
  if (ok) ok = mlb_run_gates(s, gates.data(), gates.size()) == MLB_OK;
  if (ok) {
    probs.resize(dim * sizeof(double));
    // re*re + im*im per amplitude, as moonlab_qgtl_execute dumps them
    ok = mlb_probabilities(s, 1, reinterpret_cast<double*>(probs.data()), nullptr) == MLB_OK;
  }
  if (s) mlb_state_free(s);
  if (!ok) {
    out = err_frame(kCtlRejected, "execute");
    return MLB_OK;
  }
  char b[64];
  std::snprintf(b, sizeof b, "OK %zu\n", dim);
  out.head = b;
  out.payload = std::move(probs);
  return MLB_OK;
}

int handle(mlb_control* c, const uint8_t* req, size_t len, Frame& out) {
  if (len == 0) {
    out = err_frame(kCtlProtocol, "empty frame");
    return MLB_OK;
  }
  const uint8_t* nl = static_cast<const uint8_t*>(std::memchr(req, '\n', len < kVerbCap ? len : kVerbCap));
  const size_t line_len = nl ? (size_t)(nl - req) : len;
  if (!nl && len >= kVerbCap) {
    out = err_frame(kCtlProtocol, "header too long");
    return MLB_OK;
  }
  char hdr[kVerbCap + 1];
  std::memcpy(hdr, req, line_len);
  hdr[line_len] = '\0';
  if (line_len == 6 && std::strncmp(hdr, "HEALTH", 6) == 0) {
    out = Frame{"OK alive\n", {}};
    return MLB_OK;
  }
  bool shots_mode = false;
  long shots = 0, body = -1;
  if (std::strncmp(hdr, "CIRCUIT ", 8) == 0) {
    if (std::sscanf(hdr + 8, "%ld", &body) != 1) {
      out = err_frame(kCtlProtocol, "expected CIRCUIT <N>");
      return MLB_OK;
    }
  } else if (std::strncmp(hdr, "SHOTS ", 6) == 0) {
    if (std::sscanf(hdr + 6, "%ld %ld", &shots, &body) != 2) {
      out = err_frame(kCtlProtocol, "expected SHOTS <shots> <bytes>");
      return MLB_OK;
    }
    if (shots <= 0 || shots > kMaxShots) {
      out = err_frame(kCtlBadArg, "shots out of range");
      return MLB_OK;
    }
    shots_mode = true;
  } else {
    out = err_frame(kCtlProtocol, "unknown verb");
    return MLB_OK;
  }
  if (body <= 0 || body > kMaxBodyBytes) {
    out = err_frame(kCtlBadArg, "body bytes out of range");
    return MLB_OK;
  }
  const size_t body_at = nl ? line_len + 1 : len;
  if (len - body_at < (size_t)body) {
    out = err_frame(kCtlProtocol, "short body");
    return MLB_OK;
  }
  uint32_t n = 0;
  size_t count = 0;
  const char* text = reinterpret_cast<const char*>(req + body_at);
  if (mlb_circuit_parse_text(text, (size_t)body, &n, nullptr, 0, &count) != MLB_OK) {
    out = err_frame(kCtlRejected, "deserialize");
    return MLB_OK;
  }
  std::vector<mlb_gate_t> gates(count);
  if (mlb_circuit_parse_text(text, (size_t)body, &n, gates.data(), count, &count) != MLB_OK) {
    out = err_frame(kCtlRejected, "deserialize");
    return MLB_OK;
  }
  if (n > c->max_qubits) {
    out = err_frame(kCtlBadArg, "qubit count exceeds server cap");
    return MLB_OK;
  }
  return shots_mode ? shots_request(c, n, gates, shots, out) : circuit_request(c, n, gates, out);
}

}  // namespace

extern "C" {

int mlb_control_create(int device, size_t hbm_budget_bytes, int num_workers, uint32_t max_qubits,
                       mlb_control_t** out) {
  if (!out) return mlb::record_error(MLB_ERR_INVALID_ARG, "null out");
  *out = nullptr;
  if (num_workers < 1 || num_workers > 256) return mlb::record_error(MLB_ERR_INVALID_ARG, "num_workers must be 1..256");
  if (max_qubits > kMaxQubitsC128) return mlb::record_error(MLB_ERR_INVALID_ARG, "max_qubits above 33");
  auto* c = new (std::nothrow) mlb_control();
  if (!c) return mlb::record_error(MLB_ERR_OUT_OF_MEMORY, "host allocation");
  c->device = device;
  c->hbm_budget = hbm_budget_bytes;
  c->num_workers = num_workers;
  c->max_qubits = max_qubits ? max_qubits : kDefaultMaxQubits;
  *out = c;
  return MLB_OK;
}

int mlb_control_set_seed(mlb_control_t* c, uint64_t seed) {
  if (!c) return mlb::record_error(MLB_ERR_INVALID_ARG, "null handle");
  c->fixed_seed = seed != 0;
  c->seed = seed;
  return MLB_OK;
}

int mlb_control_handle(mlb_control_t* c, const void* request, size_t request_len, void** response,
                       size_t* response_len) {
  if (!c || (!request && request_len) || !response || !response_len)
    return mlb::record_error(MLB_ERR_INVALID_ARG, "null argument");
  *response = nullptr;
  *response_len = 0;
  Frame f;
  handle(c, static_cast<const uint8_t*>(request), request_len, f);
  const size_t total = f.head.size() + f.payload.size();
  auto* buf = static_cast<uint8_t*>(std::malloc(total ? total : 1));
  if (!buf) return mlb::record_error(MLB_ERR_OUT_OF_MEMORY, "response allocation");
  std::memcpy(buf, f.head.data(), f.head.size());
  if (!f.payload.empty()) std::memcpy(buf + f.head.size(), f.payload.data(), f.payload.size());
  *response = buf;
  *response_len = total;
  return MLB_OK;
}

void mlb_control_free(void* response) { std::free(response); }

void mlb_control_destroy(mlb_control_t* c) {
  if (!c) return;
  if (c->server) mlb_server_destroy(c->server);
  delete c;
}

}  // extern "C"
