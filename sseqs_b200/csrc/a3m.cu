// Host-side a3m row assembly (sseqs/to_a3m.py:16-72): the rows of the a3m
// file built from traceback results, in a given order, with the reference's
// placement, case and filtering rules.  Plain C++ (no device code); the
// Python layer computes the order (np.argsort of the scores, descending) and
// passes pointers into the traceback's host byte matrices.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_set>

#include "sseqs_b200.h"

namespace {
inline char upper_ascii(uint8_t c) { return (char)((c >= 'a' && c <= 'z') ? c - 32 : c); }
inline char lower_ascii(uint8_t c) { return (char)((c >= 'A' && c <= 'Z') ? c + 32 : c); }
}  // namespace

extern "C" int sseqs_a3m_rows(const char* query, int64_t query_len, int64_t n_rows,
                              const int64_t* order, const uint8_t* const* q_rows,
                              const uint8_t* const* t_rows, const int32_t* lens,
                              const int64_t* scores, char* out, int64_t out_cap,
                              int64_t* out_len) {
  if (!query || query_len < 0 || n_rows < 0 || !out || !out_len || out_cap < 0 ||
      (n_rows > 0 && (!order || !q_rows || !t_rows || !lens || !scores)))
    return SSEQS_ERR_ARG;
  *out_len = 0;
  const std::string q(query, (size_t)query_len);
  std::unordered_set<std::string> seen;
  seen.reserve((size_t)n_rows * 2 + 1);
  std::string compact, row;
  char head[64];
  int64_t pos = 0;
  for (int64_t i = 0; i < n_rows; ++i) {
    const int64_t k = order[i];
    if (k < 0 || k >= n_rows) return SSEQS_ERR_ARG;
    const int32_t n = lens[k];
    if (scores[k] == 0 || n <= 0) continue;          // score 0 or no alignment
    const uint8_t* qa = q_rows[k];
    const uint8_t* ta = t_rows[k];
    compact.clear();
    for (int32_t j = 0; j < n; ++j)
      if (qa[j] != '-') compact.push_back((char)qa[j]);
    const size_t q0 = q.find(compact);               // first occurrence, as str.find
    if (q0 == std::string::npos) return SSEQS_ERR_UNSUPPORTED;
    row.assign(q0, '-');
    bool at = false;
    for (int32_t j = 0; j < n; ++j) {
      const uint8_t tc = ta[j];
      const char c = tc == '-' ? '-' : (qa[j] != '-' ? upper_ascii(tc) : lower_ascii(tc));
      at |= c == '@';
      row.push_back(c);
    }
    row.append((size_t)query_len - q0 - compact.size(), '-');
    if (at || !seen.insert(row).second) continue;
    const int h = std::snprintf(head, sizeof head, ">target_%lld score=%lld.0\n", (long long)i,
                                (long long)scores[k]);
    if (h <= 0 || pos + h + (int64_t)row.size() + 1 > out_cap) return SSEQS_ERR_CAPACITY;
    std::memcpy(out + pos, head, (size_t)h);
    pos += h;
    std::memcpy(out + pos, row.data(), row.size());
    pos += (int64_t)row.size();
    out[pos++] = '\n';
  }
  *out_len = pos;
  return SSEQS_OK;
}
