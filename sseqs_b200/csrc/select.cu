// Selection primitives of the search path, all device-resident (no host
// round-trip between kernels):
//   * delimiter scan: positions of '@' in a decoded batch (sseqs/msa.py:227);
//   * segment table: per-segment lengths, the non-empty subset and its
//     running offsets (sseqs/msa.py:237-267);
//   * top-k: indices of the k largest scores with ties at the k-th value
//     taken lowest index first, returned in increasing index order -- the
//     canonical form of torch.topk + sort at sseqs/msa.py:297, 307, 324, 335.
//
// Compaction is tile-based: a tile of kTile items per block-iteration;
// pass 1 counts selected items per tile, pass 2 turns the counts into
// exclusive offsets (one block), pass 3 re-evaluates the predicate and writes
// each selected item at offset + rank-in-tile (a block-wide scan), so outputs
// keep input order.  Top-k finds the exact k-th largest key with four
// 8-bit radix passes (shared-memory histograms merged with 256 global atomics
// per block) before compacting.
#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace sseqs {
namespace {

constexpr int kSelThreads = 256;
constexpr int kItems = 16;                      // items per thread and tile
constexpr int kTile = kSelThreads * kItems;     // 4096

struct TopkCtl {
  uint32_t prefix;     // key bits fixed so far
  uint32_t mask;       // which bits of prefix are fixed
  int64_t kleft;       // elements still to take at or below the prefix
  uint32_t hist[256];
};

// Block-wide exclusive scan of one int64 per thread; returns the total.
__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* out_excl) {
  __shared__ int64_t warp_sums[kSelThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int64_t s = (lane < kSelThreads / 32) ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kSelThreads / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  const int64_t before = (wid == 0 ? 0 : warp_sums[wid - 1]) + x - v;
  const int64_t total = warp_sums[kSelThreads / 32 - 1];
  __syncthreads();
  *out_excl = before;
  return total;
}

// ------------------------------------------------------------ predicates
struct IsByte {
  const uint8_t* p;
  uint8_t v;
  __device__ bool operator()(int64_t i) const { return p[i] == v; }
};
struct NonZero {
  const int32_t* p;
  __device__ bool operator()(int64_t i) const { return p[i] != 0; }
};

template <class Pred>
__global__ void __launch_bounds__(kSelThreads) count_kernel(Pred pred, int64_t n, int64_t* cnt) {
  const int64_t ntile = (n + kTile - 1) / kTile;
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int64_t b = tile * kTile;
    int c = 0;
#pragma unroll 4
    for (int i = 0; i < kItems; ++i) {
      const int64_t x = b + (int64_t)i * kSelThreads + threadIdx.x;
      if (x < n && pred(x)) ++c;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    __shared__ int ws[kSelThreads / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t s = 0;
      for (int w = 0; w < kSelThreads / 32; ++w) s += ws[w];
      cnt[tile] = s;
    }
    __syncthreads();
  }
}

// Exclusive scan of cnt[0..m) in place (one block); total -> *total.
__global__ void __launch_bounds__(kSelThreads) scan_counts_kernel(int64_t* cnt, int64_t m, int64_t* total) {
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < m; base += kSelThreads) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = i < m ? cnt[i] : 0;
    int64_t ex;
    const int64_t tot = block_exclusive_scan(v, &ex);
    if (i < m) cnt[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

// Writes index i (as int32) of every selected item at its compacted slot;
// with `vals`, also writes vals[i].
template <class Pred>
__global__ void __launch_bounds__(kSelThreads)
    scatter_kernel(Pred pred, int64_t n, const int64_t* off, int32_t* out_idx, int64_t max_out,
                   const int32_t* vals, int32_t* out_vals) {
  const int64_t ntile = (n + kTile - 1) / kTile;
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    // thread-contiguous items keep the output in input order
    const int64_t b = tile * kTile + (int64_t)threadIdx.x * kItems;
    uint32_t bits = 0;
    int c = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      const int64_t x = b + i;
      if (x < n && pred(x)) { bits |= 1u << i; ++c; }
    }
    int64_t ex;
    block_exclusive_scan(c, &ex);
    int64_t o = off[tile] + ex;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      if (bits & (1u << i)) {
        if (o < max_out) {
          out_idx[o] = (int32_t)(b + i);
          if (vals) out_vals[o] = vals[b + i];
        }
        ++o;
      }
    }
  }
}

// -------------------------------------------------------------- top-k
template <int KT>
__device__ __forceinline__ uint32_t key_of(const void* keys, int64_t i) {
  if constexpr (KT == 0) {   // int32 -> order-preserving unsigned
    return (uint32_t)reinterpret_cast<const int32_t*>(keys)[i] ^ 0x80000000u;
  } else {                   // IEEE half bits -> order-preserving unsigned
    const uint32_t h = reinterpret_cast<const uint16_t*>(keys)[i];
    return (h & 0x8000u) ? (~h & 0xffffu) : (h | 0x8000u);
  }
}

__global__ void topk_init_kernel(TopkCtl* ctl, int64_t k) {
  for (int i = threadIdx.x; i < 256; i += blockDim.x) ctl->hist[i] = 0;
  if (threadIdx.x == 0) {
    ctl->prefix = 0;
    ctl->mask = 0;
    ctl->kleft = k;
  }
}

template <int KT>
__global__ void __launch_bounds__(kSelThreads)
    topk_hist_kernel(const void* keys, int64_t n, TopkCtl* ctl, int shift) {
  __shared__ uint32_t h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const uint32_t prefix = ctl->prefix, mask = ctl->mask;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = key_of<KT>(keys, i);
    if ((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(&ctl->hist[i], h[i]);
}

__global__ void topk_pick_kernel(TopkCtl* ctl, int shift) {
  if (threadIdx.x == 0) {
    int64_t above = 0;
    int d = 255;
    for (; d > 0; --d) {
      const int64_t c = ctl->hist[d];
      if (above + c >= ctl->kleft) break;
      above += c;
    }
    ctl->prefix |= (uint32_t)d << shift;
    ctl->mask |= 255u << shift;
    ctl->kleft -= above;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x) ctl->hist[i] = 0;
}

template <int KT>
__global__ void __launch_bounds__(kSelThreads)
    topk_count_kernel(const void* keys, int64_t n, const TopkCtl* ctl, int64_t* cnt_gt, int64_t* cnt_eq) {
  const uint32_t T = ctl->prefix;
  const int64_t ntile = (n + kTile - 1) / kTile;
  __shared__ int wg[kSelThreads / 32], we[kSelThreads / 32];
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int64_t b = tile * kTile + (int64_t)threadIdx.x * kItems;
    int g = 0, e = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      if (b + i < n) {
        const uint32_t k = key_of<KT>(keys, b + i);
        g += k > T;
        e += k == T;
      }
    }
    g = __reduce_add_sync(0xffffffffu, g);
    e = __reduce_add_sync(0xffffffffu, e);
    if ((threadIdx.x & 31) == 0) { wg[threadIdx.x >> 5] = g; we[threadIdx.x >> 5] = e; }
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t sg = 0, se = 0;
      for (int w = 0; w < kSelThreads / 32; ++w) { sg += wg[w]; se += we[w]; }
      cnt_gt[tile] = sg;
      cnt_eq[tile] = se;
    }
    __syncthreads();
  }
}

template <int KT>
__global__ void __launch_bounds__(kSelThreads)
    topk_scatter_kernel(const void* keys, int64_t n, const TopkCtl* ctl, const int64_t* off_gt,
                        const int64_t* off_eq, int32_t* out_idx) {
  const uint32_t T = ctl->prefix;
  const int64_t kleft = ctl->kleft;
  const int64_t ntile = (n + kTile - 1) / kTile;
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int64_t b = tile * kTile + (int64_t)threadIdx.x * kItems;
    uint32_t gb = 0, eb = 0;
    int g = 0, e = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      if (b + i < n) {
        const uint32_t k = key_of<KT>(keys, b + i);
        if (k > T) { gb |= 1u << i; ++g; }
        else if (k == T) { eb |= 1u << i; ++e; }
      }
    }
    int64_t gx, ex;
    block_exclusive_scan(g, &gx);
    block_exclusive_scan(e, &ex);
    int64_t G = off_gt[tile] + gx, E = off_eq[tile] + ex;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      const bool isg = gb & (1u << i), ise = eb & (1u << i);
      if (isg || (ise && E < kleft)) out_idx[G + min(E, kleft)] = (int32_t)(b + i);
      G += isg;
      E += ise;
    }
  }
}

__global__ void iota_kernel(int32_t* out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int32_t)i;
}

// ------------------------------------------------------- segment table
// lengths of segments 0..nd-1 (ending at delim[k]) plus, when the batch does
// not end in '@', the trailing segment [delim[nd-1]+1, n)  (msa.py:240-247).
__global__ void seg_lengths_kernel(const int32_t* delim, const int64_t* nd_dev, int64_t n,
                                   const uint8_t* ascii, int32_t* lengths, int64_t* nseg_out) {
  const int64_t nd = *nd_dev;
  const bool trailing = (n > 0) && ascii[n - 1] != 64;
  const int64_t nseg = nd + (trailing ? 1 : 0);
  if (blockIdx.x == 0 && threadIdx.x == 0) *nseg_out = nseg;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nseg;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t prev = (k == 0) ? -1 : (int64_t)delim[k - 1];
    const int64_t end = (k < nd) ? (int64_t)delim[k] : n;
    lengths[k] = (int32_t)(end - prev - 1);
  }
}

__global__ void gather_lengths_kernel(const int32_t* lengths, const int32_t* idx, const int64_t* m_dev,
                                      int32_t* out, int64_t* offsets, int32_t* maxlen) {
  const int64_t m = *m_dev;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = lengths[idx[i]];
    out[i] = v;
    offsets[i] = v + 1;   // scanned afterwards
    atomicMax(maxlen, v);
  }
}

__global__ void exclusive_tiles_kernel(const int64_t* in, int64_t n, int64_t* tile_sum) {
  const int64_t ntile = (n + kTile - 1) / kTile;
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int64_t b = tile * kTile + (int64_t)threadIdx.x * kItems;
    int64_t s = 0;
    for (int i = 0; i < kItems; ++i)
      if (b + i < n) s += in[b + i];
    int64_t ex;
    const int64_t tot = block_exclusive_scan(s, &ex);
    if (threadIdx.x == 0) tile_sum[tile] = tot;
  }
}

__global__ void exclusive_apply_kernel(int64_t* data, int64_t n, const int64_t* tile_off) {
  const int64_t ntile = (n + kTile - 1) / kTile;
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int64_t b = tile * kTile + (int64_t)threadIdx.x * kItems;
    int64_t v[kItems];
    int64_t s = 0;
    for (int i = 0; i < kItems; ++i) {
      v[i] = (b + i < n) ? data[b + i] : 0;
      s += v[i];
    }
    int64_t ex;
    block_exclusive_scan(s, &ex);
    int64_t run = tile_off[tile] + ex;
    for (int i = 0; i < kItems; ++i)
      if (b + i < n) {
        data[b + i] = run;
        run += v[i];
      }
  }
}

// out[r][0..width) = ascii[offsets[g] + c] for c < min(width, lengths[g]),
// g = idx[r]; out_len[r] = min(width, lengths[g]).
__global__ void gather_windows_kernel(const uint8_t* ascii, const int64_t* offsets,
                                      const int32_t* lengths, const int32_t* idx, int64_t n,
                                      int width, uint8_t* out, int32_t* out_len) {
  for (int64_t r = blockIdx.x; r < n; r += gridDim.x) {
    const int32_t g = idx[r];
    const int64_t off = offsets[g];
    const int len = min(width, (int)lengths[g]);
    for (int c = threadIdx.x; c < width; c += blockDim.x)
      out[r * width + c] = c < len ? ascii[off + c] : (uint8_t)0;
    if (threadIdx.x == 0) out_len[r] = len;
  }
}

inline int grid_for(int64_t n) {
  const int64_t tiles = (n + kTile - 1) / kTile;
  return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)device_sm_count() * 8));
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace sseqs

using namespace sseqs;

// ----------------------------------------------------------- delimiters
extern "C" size_t sseqs_find_delims_workspace_bytes(int64_t n) {
  const int64_t tiles = (n + kTile - 1) / kTile;
  return align256(sizeof(int64_t) * (size_t)std::max<int64_t>(tiles, 1));
}

extern "C" int sseqs_find_delims(const uint8_t* ascii, int64_t n, int32_t* out_pos, int64_t max_out,
                                 int64_t* count, void* workspace, size_t ws_bytes,
                                 cudaStream_t stream) {
  if (n < 0 || (n > 0 && (!ascii || !count)) || max_out < 0) return SSEQS_ERR_ARG;
  if (n > INT32_MAX) return SSEQS_ERR_UNSUPPORTED;   // positions are int32 per batch
  if (!workspace || ws_bytes < sseqs_find_delims_workspace_bytes(n)) return SSEQS_ERR_WORKSPACE;
  if (n == 0) return status_of(cudaMemsetAsync(count, 0, sizeof(int64_t), stream));
  int64_t* cnt = reinterpret_cast<int64_t*>(workspace);
  const int64_t tiles = (n + kTile - 1) / kTile;
  const int grid = grid_for(n);
  IsByte pred{ascii, 64};
  { count_kernel<<<grid, kSelThreads, 0, stream>>>(pred, n, cnt); count_launches(1); }
  { scan_counts_kernel<<<1, kSelThreads, 0, stream>>>(cnt, tiles, count); count_launches(1); }
  { scatter_kernel<<<grid, kSelThreads, 0, stream>>>(pred, n, cnt, out_pos, max_out, nullptr, nullptr); count_launches(1); }
  return status_of(cudaGetLastError());
}

// ---------------------------------------------------------- segment table
extern "C" size_t sseqs_segment_table_workspace_bytes(int64_t max_segments) {
  const int64_t tiles = (max_segments + kTile - 1) / kTile;
  return align256(sizeof(int32_t) * (size_t)std::max<int64_t>(max_segments, 1)) +
         2 * align256(sizeof(int64_t) * (size_t)std::max<int64_t>(tiles, 1)) + 256;
}

extern "C" int sseqs_segment_table(const uint8_t* ascii, int64_t n, const int32_t* delim,
                                   const int64_t* n_delims, int64_t max_segments, int32_t* seg_index,
                                   int32_t* lengths, int64_t* offsets, int64_t* n_segments,
                                   int32_t* maxlen, void* workspace, size_t ws_bytes,
                                   cudaStream_t stream) {
  if (n < 0 || max_segments < 1 || !ascii || !delim || !n_delims || !seg_index || !lengths ||
      !offsets || !n_segments || !maxlen)
    return SSEQS_ERR_ARG;
  if (!workspace || ws_bytes < sseqs_segment_table_workspace_bytes(max_segments))
    return SSEQS_ERR_WORKSPACE;
  char* ws = reinterpret_cast<char*>(workspace);
  int32_t* all_len = reinterpret_cast<int32_t*>(ws);
  ws += align256(sizeof(int32_t) * (size_t)max_segments);
  const int64_t tiles = (max_segments + kTile - 1) / kTile;
  int64_t* cnt = reinterpret_cast<int64_t*>(ws);
  ws += align256(sizeof(int64_t) * (size_t)std::max<int64_t>(tiles, 1));
  int64_t* tsum = reinterpret_cast<int64_t*>(ws);
  ws += align256(sizeof(int64_t) * (size_t)std::max<int64_t>(tiles, 1));
  int64_t* nall = reinterpret_cast<int64_t*>(ws);
  const int grid = grid_for(max_segments);
  // The segment count is only known on the device; the passes below run over
  // max_segments slots, so the slots past the real count are cleared to read
  // as empty (seg_lengths_kernel writes only [0, nseg)).
  cudaMemsetAsync(all_len, 0, sizeof(int32_t) * (size_t)max_segments, stream);
  cudaMemsetAsync(maxlen, 0, sizeof(int32_t), stream);
  // all segments (the reference's `lengths` before filtering)
  { seg_lengths_kernel<<<grid, kSelThreads, 0, stream>>>(delim, n_delims, n, ascii, all_len, nall); count_launches(1); }
  NonZero nz{all_len};
  { count_kernel<<<grid, kSelThreads, 0, stream>>>(nz, max_segments, cnt); count_launches(1); }
  { scan_counts_kernel<<<1, kSelThreads, 0, stream>>>(cnt, tiles, n_segments); count_launches(1); }
  { scatter_kernel<<<grid, kSelThreads, 0, stream>>>(nz, max_segments, cnt, seg_index, max_segments,
                                                  nullptr, nullptr); count_launches(1); }
  { gather_lengths_kernel<<<grid, kSelThreads, 0, stream>>>(all_len, seg_index, n_segments, lengths,
                                                         offsets, maxlen); count_launches(1); }
  { exclusive_tiles_kernel<<<grid, kSelThreads, 0, stream>>>(offsets, max_segments, tsum); count_launches(1); }
  { scan_counts_kernel<<<1, kSelThreads, 0, stream>>>(tsum, tiles, nullptr); count_launches(1); }
  { exclusive_apply_kernel<<<grid, kSelThreads, 0, stream>>>(offsets, max_segments, tsum); count_launches(1); }
  return status_of(cudaGetLastError());
}

// ------------------------------------------------------------------ top-k
extern "C" size_t sseqs_topk_workspace_bytes(int64_t n) {
  const int64_t tiles = (n + kTile - 1) / kTile;
  return align256(sizeof(TopkCtl)) + 2 * align256(sizeof(int64_t) * (size_t)std::max<int64_t>(tiles, 1));
}

extern "C" int sseqs_topk(const void* keys, int key_type, int64_t n, int64_t k, int32_t* out_idx,
                          void* workspace, size_t ws_bytes, cudaStream_t stream) {
  if (n < 0 || k < 0 || k > n || (key_type != 0 && key_type != 1)) return SSEQS_ERR_ARG;
  if (k == 0) return SSEQS_OK;
  if (!keys || !out_idx) return SSEQS_ERR_ARG;
  if (n > INT32_MAX) return SSEQS_ERR_UNSUPPORTED;
  if (k == n) {
    { iota_kernel<<<grid_for(n), kSelThreads, 0, stream>>>(out_idx, n); count_launches(1); }
    return status_of(cudaGetLastError());
  }
  if (!workspace || ws_bytes < sseqs_topk_workspace_bytes(n)) return SSEQS_ERR_WORKSPACE;
  char* ws = reinterpret_cast<char*>(workspace);
  TopkCtl* ctl = reinterpret_cast<TopkCtl*>(ws);
  ws += align256(sizeof(TopkCtl));
  const int64_t tiles = (n + kTile - 1) / kTile;
  int64_t* cg = reinterpret_cast<int64_t*>(ws);
  ws += align256(sizeof(int64_t) * (size_t)tiles);
  int64_t* ce = reinterpret_cast<int64_t*>(ws);
  const int grid = grid_for(n);
  const int hgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + kSelThreads - 1) / kSelThreads,
                                                                (int64_t)device_sm_count() * 4));
  { topk_init_kernel<<<1, 256, 0, stream>>>(ctl, k); count_launches(1); }
  const int first_shift = key_type == 0 ? 24 : 8;
  for (int shift = first_shift; shift >= 0; shift -= 8) {
    if (key_type == 0)
      { topk_hist_kernel<0><<<hgrid, kSelThreads, 0, stream>>>(keys, n, ctl, shift); count_launches(1); }
    else
      { topk_hist_kernel<1><<<hgrid, kSelThreads, 0, stream>>>(keys, n, ctl, shift); count_launches(1); }
    { topk_pick_kernel<<<1, 256, 0, stream>>>(ctl, shift); count_launches(1); }
  }
  if (key_type == 0) { topk_count_kernel<0><<<grid, kSelThreads, 0, stream>>>(keys, n, ctl, cg, ce); count_launches(1); }
  else { topk_count_kernel<1><<<grid, kSelThreads, 0, stream>>>(keys, n, ctl, cg, ce); count_launches(1); }
  { scan_counts_kernel<<<1, kSelThreads, 0, stream>>>(cg, tiles, nullptr); count_launches(1); }
  { scan_counts_kernel<<<1, kSelThreads, 0, stream>>>(ce, tiles, nullptr); count_launches(1); }
  if (key_type == 0) { topk_scatter_kernel<0><<<grid, kSelThreads, 0, stream>>>(keys, n, ctl, cg, ce, out_idx); count_launches(1); }
  else { topk_scatter_kernel<1><<<grid, kSelThreads, 0, stream>>>(keys, n, ctl, cg, ce, out_idx); count_launches(1); }
  return status_of(cudaGetLastError());
}

// ------------------------------------------------------------ hit windows
extern "C" int sseqs_gather_windows(const uint8_t* ascii, const int64_t* offsets,
                                    const int32_t* lengths, const int32_t* idx, int64_t n,
                                    int width, uint8_t* out, int32_t* out_len,
                                    cudaStream_t stream) {
  if (n < 0 || width < 0) return SSEQS_ERR_ARG;
  if (n == 0 || width == 0) return SSEQS_OK;
  if (!ascii || !offsets || !lengths || !idx || !out || !out_len) return SSEQS_ERR_ARG;
  const int grid = (int)std::min<int64_t>(n, (int64_t)device_sm_count() * 16);
  { gather_windows_kernel<<<grid, 128, 0, stream>>>(ascii, offsets, lengths, idx, n, width, out,
                                                  out_len); count_launches(1); }
  return status_of(cudaGetLastError());
}

// ------------------------------------------------------ segment packing
// Segment i (bytes [src[i], src[i] + len[i]) of the buffer bases[part[i]])
// goes to out[dst[i] ..], followed by one '@'.  One warp per segment: the
// bytes are moved as 4-byte words where source and destination share their
// alignment, else byte by byte.
__global__ void pack_segments_kernel(const uint64_t* bases, const int32_t* part,
                                     const int64_t* src, const int32_t* len, const int64_t* dst,
                                     int64_t n, uint8_t* out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const uint8_t* s = reinterpret_cast<const uint8_t*>(bases[part[i]]) + src[i];
    uint8_t* d = out + dst[i];
    const int L = len[i];
    const int head = (int)((4 - (reinterpret_cast<uintptr_t>(d) & 3)) & 3);
    if (((reinterpret_cast<uintptr_t>(s) ^ reinterpret_cast<uintptr_t>(d)) & 3) == 0 && L > head) {
      if (lane < head) d[lane] = s[lane];
      const int words = (L - head) >> 2;
      const uint32_t* sw = reinterpret_cast<const uint32_t*>(s + head);
      uint32_t* dw = reinterpret_cast<uint32_t*>(d + head);
      for (int w = lane; w < words; w += 32) dw[w] = sw[w];
      for (int b = head + 4 * words + lane; b < L; b += 32) d[b] = s[b];
    } else {
      for (int b = lane; b < L; b += 32) d[b] = s[b];
    }
    if (lane == 0) d[L] = 64;
  }
}

extern "C" int sseqs_pack_segments(const uint64_t* bases, const int32_t* part, const int64_t* src,
                                   const int32_t* len, const int64_t* dst, int64_t n, uint8_t* out,
                                   cudaStream_t stream) {
  if (n < 0) return SSEQS_ERR_ARG;
  if (n == 0) return SSEQS_OK;
  if (!bases || !part || !src || !len || !dst || !out) return SSEQS_ERR_ARG;
  const int grid = (int)std::min<int64_t>((n + 7) / 8, (int64_t)device_sm_count() * 16);
  { pack_segments_kernel<<<grid, 256, 0, stream>>>(bases, part, src, len, dst, n, out);
    count_launches(1); }
  return status_of(cudaGetLastError());
}

// ------------------------------------------------ top-k without allocation
// Scratch of sseqs_topk_static: the same control block and per-tile counters
// as sseqs_topk's workspace, in a fixed array that every GPU loading this
// library holds until the process exits (about 66 KB).  Host code may not
// pass this symbol to a kernel (on the host it names a stand-in, not device
// memory); it uses the device address fetched below.
namespace {
constexpr int64_t kStaticTopkMaxN = SSEQS_TOPK_STATIC_MAX_N;
constexpr int64_t kStaticTopkTiles = kStaticTopkMaxN / kTile;
constexpr size_t kStaticCtlBytes = (sizeof(TopkCtl) + 255) & ~(size_t)255;
constexpr size_t kStaticScratchBytes =
    kStaticCtlBytes + 2 * sizeof(int64_t) * (size_t)kStaticTopkTiles;
static_assert(kStaticTopkMaxN % kTile == 0, "capacity must be whole tiles");

static __device__ __align__(256) unsigned char g_topk_scratch[kStaticScratchBytes];

// Device address of g_topk_scratch for the current device, looked up once
// per device (with that device current) and cached.
int static_topk_scratch(unsigned char** out) {
  static std::mutex mu;
  static unsigned char* addr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SSEQS_ERR_CUDA;
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_topk_scratch) != cudaSuccess || !p) return SSEQS_ERR_CUDA;
    addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = addr[dev];
  return SSEQS_OK;
}
}  // namespace

extern "C" int sseqs_topk_static(const void* keys, int key_type, int64_t n, int64_t k,
                                 int32_t* out_idx, cudaStream_t stream) {
  if (n < 0 || k < 0 || k > n || (key_type != 0 && key_type != 1)) return SSEQS_ERR_ARG;
  if (n > kStaticTopkMaxN) return SSEQS_ERR_CAPACITY;
  if (k == 0) return SSEQS_OK;
  if (!keys || !out_idx) return SSEQS_ERR_ARG;
  if (k == n) {
    { iota_kernel<<<grid_for(n), kSelThreads, 0, stream>>>(out_idx, n); count_launches(1); }
    return status_of(cudaGetLastError());
  }
  unsigned char* base = nullptr;
  const int st = static_topk_scratch(&base);
  if (st != SSEQS_OK) return st;
  // The control block is rewritten by topk_init_kernel at the start of every
  // call, and every counter slot a call reads is written earlier in the same
  // call, so nothing left over from a previous call is read.
  TopkCtl* ctl = reinterpret_cast<TopkCtl*>(base);
  int64_t* cg = reinterpret_cast<int64_t*>(base + kStaticCtlBytes);
  int64_t* ce = cg + kStaticTopkTiles;
  const int64_t tiles = (n + kTile - 1) / kTile;
  const int grid = grid_for(n);
  const int hgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + kSelThreads - 1) / kSelThreads,
                                                                (int64_t)device_sm_count() * 4));
  { topk_init_kernel<<<1, 256, 0, stream>>>(ctl, k); count_launches(1); }
  const int first_shift = key_type == 0 ? 24 : 8;
  for (int shift = first_shift; shift >= 0; shift -= 8) {
    if (key_type == 0)
      { topk_hist_kernel<0><<<hgrid, kSelThreads, 0, stream>>>(keys, n, ctl, shift); count_launches(1); }
    else
      { topk_hist_kernel<1><<<hgrid, kSelThreads, 0, stream>>>(keys, n, ctl, shift); count_launches(1); }
    { topk_pick_kernel<<<1, 256, 0, stream>>>(ctl, shift); count_launches(1); }
  }
  if (key_type == 0) { topk_count_kernel<0><<<grid, kSelThreads, 0, stream>>>(keys, n, ctl, cg, ce); count_launches(1); }
  else { topk_count_kernel<1><<<grid, kSelThreads, 0, stream>>>(keys, n, ctl, cg, ce); count_launches(1); }
  { scan_counts_kernel<<<1, kSelThreads, 0, stream>>>(cg, tiles, nullptr); count_launches(1); }
  { scan_counts_kernel<<<1, kSelThreads, 0, stream>>>(ce, tiles, nullptr); count_launches(1); }
  if (key_type == 0) { topk_scatter_kernel<0><<<grid, kSelThreads, 0, stream>>>(keys, n, ctl, cg, ce, out_idx); count_launches(1); }
  else { topk_scatter_kernel<1><<<grid, kSelThreads, 0, stream>>>(keys, n, ctl, cg, ce, out_idx); count_launches(1); }
  return status_of(cudaGetLastError());
}
