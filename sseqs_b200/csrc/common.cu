// Library-wide entry points: status text, ABI version, launch counter.
#include <atomic>

#include "common.cuh"

namespace sseqs {
namespace {
std::atomic<long long> g_launches{0};
}
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace sseqs

extern "C" const char* sseqs_status_string(int status) {
  switch (status) {
    case SSEQS_OK: return "ok";
    case SSEQS_ERR_ARG: return "invalid argument";
    case SSEQS_ERR_UNSUPPORTED: return "input outside the supported range";
    case SSEQS_ERR_CUDA: return "CUDA runtime error";
    case SSEQS_ERR_WORKSPACE: return "workspace missing or too small";
    case SSEQS_ERR_CAPACITY:
      return "input larger than the fixed scratch capacity of this entry point";
    default: return "unknown status";
  }
}

extern "C" int sseqs_version(void) { return 1; }

extern "C" int64_t sseqs_launch_count(void) { return sseqs::g_launches.load(); }
