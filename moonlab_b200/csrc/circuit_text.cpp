// circuit_text.cpp -- the "moonlab-circuit v1" line format of the reference's
// QGTL ingestion surface, read straight into engine gate records and written
// back byte for byte.
//
// Reference: src/applications/moonlab_qgtl_backend.h:190-205 (the format),
// moonlab_qgtl_backend.c:319-368 (serialize), :370-406 (line scanner) and
// :414-506 (deserialize), gate names and arity :72-84, :262-298, record
// checks in moonlab_qgtl_add_gate :87-117.
//
// Format: an optional comment header, "NUM_QUBITS <n>" (1..32) as the first
// line that is not blank and not a comment, then one gate per line:
//   <NAME> <target>              I X Y Z H S T
//   <NAME> <target> <theta>      RX RY RZ (theta printed with %.17g)
//   <NAME> <target> <control>    CNOT CY CZ SWAP
// Lines are '\n'-terminated; leading whitespace is skipped; a line whose
// first non-blank character is '#' is a comment.  The reference scans each
// line with sscanf: trailing text after the fields is ignored, and the name
// is the whole first non-blank run.  This reader splits lines and matches
// names itself and reads the number fields with the same scanner, so it
// gives the same records for the same text, without building an
// intermediate circuit object.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "moonlab_b200.h"
#include "mlb_internal.h"

namespace {

constexpr size_t kLineCap = 256;  // the reference's line buffer: longer lines are invalid

const char* const kNames[14] = {"I", "X", "Y", "Z", "H", "S", "T", "RX", "RY", "RZ", "CNOT", "CY", "CZ", "SWAP"};

inline bool is_space(char c) {  // isspace in the C locale
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}
inline bool takes_theta(int t) { return t >= 7 && t <= 9; }
inline bool two_qubit(int t) { return t >= 10 && t <= 13; }

// Number fields are read with the C library's own scanner (%d, %lf), as the
// reference reads them, so edge cases agree: "0x" or "infin" is no number,
// trailing text is ignored, and an int field out of range converts as the
// library converts it.  Advances p.
bool read_int(const char*& p, int& out) {
  int used = 0;
  if (std::sscanf(p, "%d%n", &out, &used) != 1) return false;
  p += used;
  return true;
}

bool read_double(const char*& p, double& out) {
  int used = 0;
  if (std::sscanf(p, "%lf%n", &out, &used) != 1) return false;
  p += used;
  return true;
}

// One gate line (left-trimmed, NUL-terminated) into a record.
bool parse_gate_line(const char* line, int n, mlb_gate_t& g) {
  const char* p = line;
  const char* name = p;
  while (*p && !is_space(*p)) p++;
  const size_t len = (size_t)(p - name);
  int type = -1;
  for (int t = 0; t < 14; t++)
    if (std::strlen(kNames[t]) == len && std::memcmp(kNames[t], name, len) == 0) type = t;
  if (type < 0) return false;
  g = mlb_gate_t{};
  g.type = type;
  g.control = -1;
  if (!read_int(p, g.target) || g.target < 0 || g.target >= n) return false;
  if (two_qubit(type)) {
    if (!read_int(p, g.control) || g.control < 0 || g.control >= n || g.control == g.target) return false;
  } else if (takes_theta(type)) {
    if (!read_double(p, g.theta)) return false;
  }
  return true;
}

int parse_text(const char* text, size_t len, uint32_t& n_out, std::vector<mlb_gate_t>& gates) {
  if (len == 0) len = std::strlen(text);
  else if (std::memchr(text, '\0', len)) return MLB_ERR_INVALID_ARG;  // NUL inside the declared extent
  const char* p = text;
  const char* end = text + len;
  char line[kLineCap];
  int n = -1;
  while (p < end) {
    const char* eol = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
    if (!eol) eol = end;
    const char* s = p;
    p = eol < end ? eol + 1 : end;
    while (s < eol && is_space(*s)) s++;
    if (s == eol || *s == '#') continue;  // blank or comment
    const size_t w = (size_t)(eol - s);
    if (w + 1 > kLineCap) return MLB_ERR_INVALID_ARG;
    std::memcpy(line, s, w);  // the scanner reads NUL-terminated text
    line[w] = '\0';
    if (n < 0) {
      static const char kHead[] = "NUM_QUBITS";
      if (std::strncmp(line, kHead, sizeof kHead - 1) != 0) return MLB_ERR_INVALID_ARG;
      const char* q = line + sizeof kHead - 1;
      int v = 0;
      if (!read_int(q, v) || v < 1 || v > 32) return MLB_ERR_INVALID_ARG;
      n = v;
      continue;
    }
    mlb_gate_t g;
    if (!parse_gate_line(line, n, g)) return MLB_ERR_INVALID_ARG;
    gates.push_back(g);
  }
  if (n < 0) return MLB_ERR_INVALID_ARG;  // no header
  n_out = (uint32_t)n;
  return MLB_OK;
}

}  // namespace

extern "C" {

int mlb_circuit_parse_text(const char* text, size_t len, uint32_t* num_qubits, mlb_gate_t* gates,
                           size_t capacity, size_t* num_gates) {
  if (!text || !num_qubits || !num_gates) return mlb::record_error(MLB_ERR_INVALID_ARG, "null argument");
  std::vector<mlb_gate_t> g;
  uint32_t n = 0;
  if (parse_text(text, len, n, g) != MLB_OK)
    return mlb::record_error(MLB_ERR_INVALID_ARG, "text is not a moonlab-circuit v1 circuit");
  *num_qubits = n;
  *num_gates = g.size();
  if (!gates) return MLB_OK;
  if (capacity < g.size()) return mlb::record_error(MLB_ERR_INVALID_ARG, "gate buffer too small");
  if (!g.empty()) std::memcpy(gates, g.data(), g.size() * sizeof(mlb_gate_t));
  return MLB_OK;
}

int mlb_circuit_format_text(uint32_t num_qubits, const mlb_gate_t* gates, size_t num_gates, char* buf,
                            size_t capacity, size_t* written) {
  if ((!gates && num_gates) || (!buf && capacity) || !written)
    return mlb::record_error(MLB_ERR_INVALID_ARG, "null argument");
  std::string out = "# moonlab-circuit v1\n";
  char tmp[96];
  std::snprintf(tmp, sizeof tmp, "NUM_QUBITS %d\n", (int)num_qubits);
  out += tmp;
  for (size_t i = 0; i < num_gates; i++) {
    const mlb_gate_t& g = gates[i];
    if (g.type < 0 || g.type > 13) {
      std::snprintf(tmp, sizeof tmp, "gate %zu: type %d has no name in the text format", i, (int)g.type);
      return mlb::record_error(MLB_ERR_NOT_SUPPORTED, tmp);
    }
    if (two_qubit(g.type)) std::snprintf(tmp, sizeof tmp, "%s %d %d\n", kNames[g.type], g.target, g.control);
    else if (takes_theta(g.type)) std::snprintf(tmp, sizeof tmp, "%s %d %.17g\n", kNames[g.type], g.target, g.theta);
    else std::snprintf(tmp, sizeof tmp, "%s %d\n", kNames[g.type], g.target);
    out += tmp;
  }
  *written = out.size();
  if (!buf) return MLB_OK;  // size query
  if (capacity < out.size() + 1) {
    *written = out.size() + 1;
    return mlb::record_error(MLB_ERR_INVALID_ARG, "text buffer too small");
  }
  std::memcpy(buf, out.c_str(), out.size() + 1);
  return MLB_OK;
}

}  // extern "C"
