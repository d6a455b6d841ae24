// xbit 5-bit codec (layout of sseqs/xbit.cu:8-62): 8 symbols per 5 bytes,
// first symbol in the high bits of a big-endian 40-bit window, symbol s is
// the byte s + 64.
//
// Decoding is HBM-bound (0.625 B read + 1 B written per symbol).  A block
// stages a tile of packed bytes in shared memory with 16-byte loads of the
// aligned chunks that cover it (every chunk read holds at least one byte of
// the tile, so no load leaves the caller's 16-byte chunks), then every thread
// decodes 4 groups (32 symbols) and writes them as two 16-byte stores.
#include <algorithm>

#include "common.cuh"

namespace sseqs {
namespace {

constexpr int kDecThreads = 256;
constexpr int kGroupsPerThread = 4;                                // 32 symbols
constexpr int kTileGroups = kDecThreads * kGroupsPerThread;        // 1024 groups
constexpr int kTileBytes = kTileGroups * 5;                        // 5120 B in
constexpr int kTileChunks = kTileBytes / 16 + 2;                   // staged chunks

__device__ __forceinline__ void decode_group(const uint8_t* p, uint32_t& lo, uint32_t& hi) {
  const uint64_t w = ((uint64_t)p[0] << 32) | ((uint64_t)p[1] << 24) | ((uint64_t)p[2] << 16) |
                     ((uint64_t)p[3] << 8) | (uint64_t)p[4];
  uint32_t b[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) b[k] = (uint32_t)((w >> (35 - 5 * k)) & 31u) + 64u;
  lo = b[0] | (b[1] << 8) | (b[2] << 16) | (b[3] << 24);
  hi = b[4] | (b[5] << 8) | (b[6] << 16) | (b[7] << 24);
}

// in: packed stream starting at symbol 0; n_groups_total = ceil(n_syms / 8)
template <bool kAlignedOut>
__global__ void __launch_bounds__(kDecThreads)
    xbit_decode_kernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int64_t n_syms) {
  __shared__ uint4 stage[kTileChunks];
  const uint8_t* sbytes = reinterpret_cast<const uint8_t*>(stage);
  const int64_t n_groups = (n_syms + 7) / 8;
  const int64_t n_tiles = (n_groups + kTileGroups - 1) / kTileGroups;
  const uintptr_t iu = reinterpret_cast<uintptr_t>(in);
  const uint4* abase = reinterpret_cast<const uint4*>(iu & ~(uintptr_t)15);
  const int64_t ioff = (int64_t)(iu & 15);

  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int64_t g0 = tile * kTileGroups;
    const int64_t ng = min((int64_t)kTileGroups, n_groups - g0);
    const int64_t byte0 = g0 * 5 + ioff;          // aligned coordinates
    // exclusive end, clipped to the packed stream's (5n+7)/8 bytes
    const int64_t byte1 = min((g0 + ng) * 5, (n_syms * 5 + 7) / 8) + ioff;
    const int64_t c0 = byte0 >> 4, c1 = (byte1 + 15) >> 4;
    __syncthreads();
    for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) stage[c - c0] = __ldg(abase + c);
    __syncthreads();
    const int64_t sh = byte0 - (c0 << 4);
    const int64_t gl0 = (int64_t)threadIdx.x * kGroupsPerThread;
    uint32_t w[2 * kGroupsPerThread];
#pragma unroll
    for (int i = 0; i < kGroupsPerThread; ++i) {
      if (gl0 + i < ng) decode_group(sbytes + sh + (gl0 + i) * 5, w[2 * i], w[2 * i + 1]);
      else w[2 * i] = w[2 * i + 1] = 0;
    }
    const int64_t s0 = (g0 + gl0) * 8;            // first symbol of this thread
    if (kAlignedOut && s0 + 32 <= n_syms) {
      uint4* o = reinterpret_cast<uint4*>(out + s0);
      o[0] = make_uint4(w[0], w[1], w[2], w[3]);
      o[1] = make_uint4(w[4], w[5], w[6], w[7]);
    } else {
      for (int k = 0; k < 32 && s0 + k < n_syms; ++k) out[s0 + k] = (uint8_t)(w[k >> 2] >> ((k & 3) * 8));
    }
  }
}

__global__ void xbit_encode_kernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out,
                                   int64_t n_syms) {
  const int64_t n_groups = (n_syms + 7) / 8;
  const int64_t out_bytes = (n_syms * 5 + 7) / 8;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n_groups;
       t += (int64_t)gridDim.x * blockDim.x) {
    uint64_t w = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint8_t s = (t * 8 + k < n_syms) ? (uint8_t)(in[t * 8 + k] - 64u) : 0;
      w |= (uint64_t)(s & 31u) << (35 - 5 * k);
    }
#pragma unroll
    for (int b = 0; b < 5; ++b)
      if (t * 5 + b < out_bytes) out[t * 5 + b] = (uint8_t)(w >> (32 - 8 * b));
  }
}

}  // namespace
}  // namespace sseqs

using namespace sseqs;

extern "C" int sseqs_xbit_decompress(const uint8_t* packed, uint8_t* out, int64_t n_syms,
                                     int64_t lo_bytes, cudaStream_t stream) {
  if (n_syms < 0 || lo_bytes < 0) return SSEQS_ERR_ARG;
  if (n_syms == 0) return SSEQS_OK;
  if (!packed || !out) return SSEQS_ERR_ARG;
  const int64_t n_groups = (n_syms + 7) / 8;
  const int64_t n_tiles = (n_groups + kTileGroups - 1) / kTileGroups;
  const int grid = (int)std::min<int64_t>(n_tiles, (int64_t)device_sm_count() * 8);
  const bool aligned = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
  if (aligned)
    { xbit_decode_kernel<true><<<grid, kDecThreads, 0, stream>>>(packed + lo_bytes, out, n_syms); count_launches(1); }
  else
    { xbit_decode_kernel<false><<<grid, kDecThreads, 0, stream>>>(packed + lo_bytes, out, n_syms); count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_xbit_compress(const uint8_t* in, uint8_t* out, int64_t n_syms,
                                   cudaStream_t stream) {
  if (n_syms < 0) return SSEQS_ERR_ARG;
  if (n_syms == 0) return SSEQS_OK;
  if (!in || !out) return SSEQS_ERR_ARG;
  const int64_t n_groups = (n_syms + 7) / 8;
  const int grid = (int)std::min<int64_t>((n_groups + 255) / 256, (int64_t)device_sm_count() * 16);
  { xbit_encode_kernel<<<grid, 256, 0, stream>>>(in, out, n_syms); count_launches(1); }
  return status_of(cudaGetLastError());
}
