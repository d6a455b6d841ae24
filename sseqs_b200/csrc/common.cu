// Library-wide entry points: status text and ABI version.
#include "common.cuh"

extern "C" const char* sseqs_status_string(int status) {
  switch (status) {
    case SSEQS_OK: return "ok";
    case SSEQS_ERR_ARG: return "invalid argument";
    case SSEQS_ERR_UNSUPPORTED: return "input outside the supported range";
    case SSEQS_ERR_CUDA: return "CUDA runtime error";
    case SSEQS_ERR_WORKSPACE: return "workspace missing or too small";
    default: return "unknown status";
  }
}

extern "C" int sseqs_version(void) { return 1; }
