// Shared definitions for the sseqs_b200 CUDA kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sseqs_b200.h"

namespace sseqs {

// Residue classes used by the score kernels.  0..19 follow the order
// ARNDCQEGHILKMFPSTWYV (the order of sseqs/sw.cu:31-53); every other byte is
// class 20 and scores -4 against any query residue (sseqs/sw.cu:128-130).
// Class 21 is an internal padding row that can never raise a score.
constexpr int kNumAA = 20;
constexpr int kClsUnknown = 20;
constexpr int kClsPad = 21;
constexpr int kNumCls = 22;
constexpr int16_t kNeg = -32768;

// BLOSUM62 in the order above (published matrix; the same values as
// sseqs/sw.cu:7-29).  Row = target residue, column = query residue; the
// matrix is symmetric.  Device code reads the constant-memory copy (a
// function-local table would be rebuilt on the stack at every call).
#define SSEQS_BLOSUM62_VALUES \
  4, -1, -2, -2, 0,  -1, -1, 0,  -2, -1, -1, -1, -1, -2, -1, 1,  0,  -3, -2, 0, \
  -1, 5, 0,  -2, -3, 1,  0,  -2, 0,  -3, -2, 2,  -1, -3, -2, -1, -1, -3, -2, -3, \
  -2, 0, 6,  1,  -3, 0,  0,  0,  1,  -3, -3, 0,  -2, -3, -2, 1,  0,  -4, -2, -3, \
  -2, -2, 1, 6,  -3, 0,  2,  -1, -1, -3, -4, -1, -3, -3, -1, 0,  -1, -4, -3, -3, \
  0, -3, -3, -3, 9,  -3, -4, -3, -3, -1, -1, -3, -1, -2, -3, -1, -1, -2, -2, -1, \
  -1, 1, 0,  0,  -3, 5,  2,  -2, 0,  -3, -2, 1,  0,  -3, -1, 0,  -1, -2, -1, -2, \
  -1, 0, 0,  2,  -4, 2,  5,  -2, 0,  -3, -3, 1,  -2, -3, -1, 0,  -1, -3, -2, -2, \
  0, -2, 0,  -1, -3, -2, -2, 6,  -2, -4, -4, -2, -3, -3, -2, 0,  -2, -2, -3, -3, \
  -2, 0, 1,  -1, -3, 0,  0,  -2, 8,  -3, -3, -1, -2, -1, -2, -1, -2, -2, 2,  -3, \
  -1, -3, -3, -3, -1, -3, -3, -4, -3, 4, 2,  -3, 1,  0,  -3, -2, -1, -3, -1, 3, \
  -1, -2, -3, -4, -1, -2, -3, -4, -3, 2, 4,  -2, 2,  0,  -3, -2, -1, -2, -1, 1, \
  -1, 2, 0,  -1, -3, 1,  1,  -2, -1, -3, -2, 5,  -1, -3, -1, 0,  -1, -3, -2, -2, \
  -1, -1, -2, -3, -1, 0, -2, -3, -2, 1,  2,  -1, 5,  0,  -2, -1, -1, -1, -1, 1, \
  -2, -3, -3, -3, -2, -3, -3, -3, -1, 0, 0,  -3, 0,  6,  -4, -2, -2, 1,  3,  -1, \
  -1, -2, -2, -1, -3, -1, -1, -2, -2, -3, -3, -1, -2, -4, 7, -1, -1, -4, -3, -2, \
  1, -1, 1,  0,  -1, 0,  0,  0,  -1, -2, -2, 0,  -1, -2, -1, 4,  1,  -3, -2, -2, \
  0, -1, 0,  -1, -1, -1, -1, -2, -2, -1, -1, -1, -1, -2, -1, 1,  5,  -2, -2, 0, \
  -3, -3, -4, -4, -2, -2, -3, -2, -2, -3, -2, -3, -1, 1, -4, -3, -2, 11, 2,  -3, \
  -2, -2, -2, -3, -2, -1, -2, -3, 2, -1, -1, -2, -1, 3,  -3, -2, -2, 2,  7,  -1, \
  0, -3, -3, -3, -1, -2, -2, -3, -3, 3, 1,  -2, 1,  -1, -2, -2, 0,  -3, -1, 4
static __constant__ int8_t kBlosum62Dev[400] = {SSEQS_BLOSUM62_VALUES};
static constexpr int8_t kBlosum62Host[400] = {SSEQS_BLOSUM62_VALUES};

__host__ __device__ inline int8_t blosum62(int a, int b) {
#ifdef __CUDA_ARCH__
  return kBlosum62Dev[a * 20 + b];
#else
  return kBlosum62Host[a * 20 + b];
#endif
}

// ASCII byte -> residue class (0..19, else 20).  Bytes >= 128 are class 20;
// the reference indexes its table with a signed char there (sseqs/sw.cu:116)
// and so has no defined result for them.
__host__ __device__ inline uint8_t ascii_class(uint8_t c) {
  switch (c) {
    case 'A': return 0;  case 'R': return 1;  case 'N': return 2;
    case 'D': return 3;  case 'C': return 4;  case 'Q': return 5;
    case 'E': return 6;  case 'G': return 7;  case 'H': return 8;
    case 'I': return 9;  case 'L': return 10; case 'K': return 11;
    case 'M': return 12; case 'F': return 13; case 'P': return 14;
    case 'S': return 15; case 'T': return 16; case 'W': return 17;
    case 'Y': return 18; case 'V': return 19;
    default: return kClsUnknown;
  }
}

// Pack two int16 lanes into the int16x2 word consumed by the DPX intrinsics.
__host__ __device__ inline uint32_t pack2(int lo, int hi) {
  return (uint32_t)(uint16_t)(int16_t)lo | ((uint32_t)(uint16_t)(int16_t)hi << 16);
}

inline int status_of(cudaError_t e) { return e == cudaSuccess ? SSEQS_OK : SSEQS_ERR_CUDA; }

// Number of SMs of the current device (cached per device ordinal).
int device_sm_count();

// Adds n to the library-wide count of kernel launches (sseqs_launch_count).
void count_launches(int n);

}  // namespace sseqs
