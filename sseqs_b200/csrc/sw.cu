// Score-only Smith-Waterman: dispatch, the exact fallback kernel and the C
// ABI.  The fast int16x2 kernel is the template in sw_kernel.cuh (see there
// for its design), instantiated per stripe width in sw_inst_*.cu.
#include <climits>
#include <mutex>

#include "sw_kernel.cuh"

namespace sseqs {

int device_sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = n > 0 ? n : 148;
  }
  return cached[dev];
}

namespace sw {
// Exact restatement for gap parameters outside the fast kernel's domain
// (linear gap > 0, affine open/extend < 0): one thread per target, cells
// stored as uint16 (linear) / int16 (affine) exactly as sseqs/sw.cu does.
__global__ void sw_generic_kernel(SwArgs a, int affine) {
  uint16_t h[kMaxQuery];
  int16_t xm[kMaxQuery], xx[kMaxQuery], xy[kMaxQuery];
  const int TPT = (a.Lq + 31) / 32;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < a.n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const Win w = window_of(a, t);
    if (!w.rows) { a.out[t] = w.res; continue; }
    int best = 0;
    for (int j = 0; j < a.Lq; ++j) { h[j] = 0; xm[j] = xx[j] = xy[j] = 0; }
    for (int64_t p = w.pos; p < w.end; ++p) {
      const int c = ascii_class(a.ascii[p]);
      if (!affine) {
        int diag = 0, left = 0;
        for (int j = 0; j < a.Lq; ++j) {
          const int s = score_of(a.q, a.Lq, c, j);
          const int up = h[j];
          if (j % TPT == 0) left = 0;
          int v = max(0, max(diag + s, max(up + a.p0, left + a.p0)));
          const uint16_t v16 = (uint16_t)v;
          diag = up;
          h[j] = v16;
          left = v16;
          best = max(best, (int)v16);
        }
      } else {
        int dm = 0, dx = 0, dy = 0, lm = 0, lx = 0;
        for (int j = 0; j < a.Lq; ++j) {
          const int s = score_of(a.q, a.Lq, c, j);
          if (j % TPT == 0) { lm = 0; lx = 0; }
          const int um = xm[j], ux = xx[j], uy = xy[j];
          const int16_t m = (int16_t)max(0, max(dm + s, max(dx + s, dy + s)));
          const int16_t x = (int16_t)max(0, max(lm - a.p0, lx - a.p1));
          const int16_t y = (int16_t)max(0, max(um - a.p0, uy - a.p1));
          dm = um; dx = ux; dy = uy;
          xm[j] = m; xx[j] = x; xy[j] = y;
          lm = m; lx = x;
          best = max(best, max((int)m, max((int)x, (int)y)));
        }
      }
    }
    a.out[t] = best;
  }
}

__global__ void fill_kernel(int32_t* out, int64_t n, int32_t v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = v;
}

// ---------------------------------------------------------------- dispatch
const Tables& tables() {
  static Tables t;
  static std::once_flag once;
  std::call_once(once, [] {
    register_1_16(t);
    register_17_32(t);
    register_33_48(t);
    register_49_64(t);
    register_1_16_def(t);
    register_17_32_def(t);
    register_33_48_def(t);
    register_49_64_def(t);
  });
  return t;
}

struct Cache {
  std::mutex mu;
  int max_blocks[2][2][kModes][64][64] = {};  // [gaps][variant][mode][TPT-1][device]
  int variant[kModes][64] = {};            // chosen variant per [mode][TPT-1]
  bool pairing[64] = {};                   // per [TPT-1]: batched affine launches pair queries
};
Cache& cache() {
  static Cache c;
  return c;
}

// Target counters of the streaming kernel: every launch takes the next slot
// of this ring and zeroes it on its stream first, so launches in flight at
// the same time (up to kTicketSlots of them) never share a counter.
constexpr int kTicketSlots = 1024;
static __device__ unsigned int g_sw_tickets[kTicketSlots];

unsigned int* ticket_slot(int dev) {
  static std::mutex mu;
  static unsigned int* base[64] = {};
  static unsigned next[64] = {};
  std::lock_guard<std::mutex> lk(mu);
  if (!base[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_sw_tickets) != cudaSuccess || !p) return nullptr;
    base[dev] = static_cast<unsigned int*>(p);
  }
  return base[dev] + (next[dev]++ % kTicketSlots);
}

// Whether a launch of `mode` passes msa()'s gap parameters, so that the
// kernel twin with those as constants (DEF) scores it.
bool default_gaps(int mode, const SwArgs& a) {
  if (mode == kLin) return a.p0 == kDefGap;
  if (mode == kBoth) return a.p0 == kDefGap && a.p1 == kDefOpen && a.p2 == kDefExt;
  return a.p0 == kDefOpen && a.p1 == kDefExt;   // kAff, kPair
}

// Launches the streaming kernel for one query (qt == nullptr; target
// counter from the ring) or for the qt->n queries of a table (counters
// a.ticket[0 .. qt->n), provided by the caller).
int launch_stream(SwArgs a, int mode, const QueryTable* qt, cudaStream_t stream) {
  const int tpt = (a.Lq + 31) / 32;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64) return SSEQS_ERR_CUDA;
  const int gaps = default_gaps(mode, a) ? 1 : 0;
  int blocks_per_sm, var;
  const KernelInfo* kp;
  {
    std::lock_guard<std::mutex> lk(cache().mu);
    var = cache().variant[mode][tpt - 1];
    kp = &tables().k[gaps][var][mode][tpt - 1];
    int& mb = cache().max_blocks[gaps][var][mode][tpt - 1][dev];
    if (mb == 0) {
      if (cudaFuncSetAttribute((const void*)kp->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kp->smem) != cudaSuccess)
        return SSEQS_ERR_CUDA;
      int nb = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)kp->fn, kp->threads,
                                                        kp->smem) != cudaSuccess || nb < 1)
        return SSEQS_ERR_CUDA;
      mb = nb;
    }
    blocks_per_sm = mb;
  }
  const KernelInfo& k = *kp;
  const int64_t full = (int64_t)device_sm_count() * blocks_per_sm;
  QueryTable none{};
  const QueryTable& table = qt ? *qt : none;
  const int ny = qt ? (mode == kPair ? (qt->n + 1) / 2 : qt->n) : 1;
  unsigned int* const tickets = a.ticket;
  // The kernel counts targets in 32 bits: launches take at most 2^30 each.
  constexpr int64_t kPiece = int64_t(1) << 30;
  for (int64_t t0 = 0; t0 < a.n; t0 += kPiece) {
    SwArgs p = a;
    p.n = std::min(kPiece, a.n - t0);
    p.out = a.out + t0;
    if (a.out2) p.out2 = a.out2 + t0;
    if (a.idx) p.idx = a.idx + t0;
    else p.g0 = (int32_t)(a.g0 + t0);
    p.ticket = qt ? tickets : ticket_slot(dev);
    if (!p.ticket) return SSEQS_ERR_CUDA;
    if (cudaMemsetAsync(p.ticket, 0, sizeof(unsigned int) * ny, stream) != cudaSuccess)
      return SSEQS_ERR_CUDA;
    const int64_t need = (p.n + k.groups_per_block - 1) / k.groups_per_block;
    const int grid = (int)std::max<int64_t>(1, std::min(full, need));
    // targets per grab: at most 64/TPT (few atomics on long rows of work),
    // and small enough that every lane group gets about 8 grabs
    const int64_t groups = (int64_t)grid * k.groups_per_block;
    p.chunk = (int)std::max<int64_t>(
        1, std::min<int64_t>(std::max(1, 64 / tpt), p.n / std::max<int64_t>(1, groups * 8)));
    { k.fn<<<dim3(grid, ny), k.threads, k.smem, stream>>>(p, table); count_launches(1); }
    const int st = status_of(cudaGetLastError());
    if (st != SSEQS_OK) return st;
  }
  return SSEQS_OK;
}

bool fast_domain(bool aff, int p0, int p1) {
  // The int16x2 kernel needs every intermediate inside int16: cells are in
  // [0, 11*2048], profile words s - open in [-16388, 11].
  return aff ? (p0 >= 0 && p0 <= 16384 && p1 >= 0 && p1 <= 16384)
             : (p0 <= 0 && p0 >= -16384);
}

int run(bool aff, SwArgs a, cudaStream_t stream) {
  if (a.n < 0 || (a.n > 0 && (!a.out || !a.starts || !a.ascii))) return SSEQS_ERR_ARG;
  if (a.n == 0) return SSEQS_OK;
  if (a.Lq < 0) return SSEQS_ERR_ARG;
  if (a.Lq > kMaxQuery) return SSEQS_ERR_UNSUPPORTED;
  if (a.Lq == 0) {   // sseqs/sw.cu:73: every result is -1
    const int grid = (int)std::min<int64_t>((a.n + 255) / 256, 4096);
    { fill_kernel<<<grid, 256, 0, stream>>>(a.out, a.n, -1); count_launches(1); }
    return status_of(cudaGetLastError());
  }
  if (!a.q) return SSEQS_ERR_ARG;
  if (fast_domain(aff, a.p0, a.p1)) return launch_stream(a, aff ? kAff : kLin, nullptr, stream);
  if (a.skip != 0) return SSEQS_ERR_UNSUPPORTED;
  const int grid = (int)std::min<int64_t>((a.n + 127) / 128, (int64_t)device_sm_count() * 4);
  { sw_generic_kernel<<<grid, 128, 0, stream>>>(a, aff ? 1 : 0); count_launches(1); }
  return status_of(cudaGetLastError());
}

// ------------------------------------------------------- DPX peak probe
__global__ void dpx_peak_kernel(uint32_t* sink, int iters, uint32_t seed) {
  uint32_t x[8], y[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    x[i] = seed * (threadIdx.x + 7 * i + 1);
    y[i] = seed ^ (blockIdx.x + 13 * i);
  }
  const uint32_t d = seed | 0x00010001u, e = seed >> 3;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      x[i] = __viaddmax_s16x2_relu(x[i], d, y[i]);
      y[i] = __vimax3_s16x2(y[i], x[i], e);
    }
  }
  uint32_t acc = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) acc ^= x[i] ^ y[i];
  if (acc == 0x9e3779b9u) sink[0] = acc;   // practically never taken
}

// int16x2 issue peak over both pipes: independent max-type DPX chains (ALU
// pipe) interleaved with int16x2 add chains (FMA pipe).
__global__ void int16x2_peak_kernel(uint32_t* sink, int iters, uint32_t seed) {
  uint32_t x[8], y[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    x[i] = seed * (threadIdx.x + 7 * i + 1);
    y[i] = seed ^ (blockIdx.x + 13 * i);
  }
  const uint32_t d = seed | 0x00010001u, e = seed >> 3;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      x[i] = __vimax3_s16x2_relu(x[i], d, e ^ (uint32_t)i);
      y[i] = __vadd2(y[i], d);
    }
  }
  uint32_t acc = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) acc ^= x[i] ^ y[i];
  if (acc == 0x9e3779b9u) sink[0] = acc;   // practically never taken
}

int time_peak(void (*kern)(uint32_t*, int, uint32_t), uint32_t* sink, double* out,
              cudaStream_t stream) {
  const int blocks = device_sm_count() * 8, threads = 256, iters = 1 << 14;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return SSEQS_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return SSEQS_ERR_CUDA; }
  { kern<<<blocks, threads, 0, stream>>>(sink, iters / 8, 0x12345u); count_launches(1); }
  cudaEventRecord(e0, stream);
  { kern<<<blocks, threads, 0, stream>>>(sink, iters, 0x12345u); count_launches(1); }
  cudaEventRecord(e1, stream);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess || ms <= 0.f) return SSEQS_ERR_CUDA;
  *out = (double)blocks * threads * iters * 16.0 / (ms * 1e-3);
  return SSEQS_OK;
}

}  // namespace sw
}  // namespace sseqs

using namespace sseqs;
using namespace sseqs::sw;

extern "C" int sseqs_max_query_len(void) { return kMaxQuery; }

extern "C" int sseqs_sw_linear(const uint8_t* query_idx, int query_len, const int32_t* good_idx,
                               const uint8_t* ascii, const int32_t* starts, int64_t n_targets,
                               int32_t* out, int gap, cudaStream_t stream) {
  if (!good_idx && n_targets > 0) return SSEQS_ERR_ARG;
  SwArgs a{query_idx, query_len, good_idx, 0, n_targets, ascii, starts, 0, out, gap, 0};
  return run(false, a, stream);
}

extern "C" int sseqs_sw_affine(const uint8_t* query_idx, int query_len, const int32_t* good_idx,
                               const uint8_t* ascii, const int32_t* starts, int64_t n_targets,
                               int32_t* out, int gap_open, int gap_extend, cudaStream_t stream) {
  if (!good_idx && n_targets > 0) return SSEQS_ERR_ARG;
  SwArgs a{query_idx, query_len, good_idx, 0, n_targets, ascii, starts, 0, out, gap_open, gap_extend};
  return run(true, a, stream);
}

extern "C" int sseqs_sw_scan(int affine, const uint8_t* query_idx, int query_len,
                             const int32_t* good_idx, int32_t g0, int64_t n_targets,
                             const uint8_t* ascii, const int32_t* delim, int skip, int32_t* out,
                             int gap_a, int gap_b, cudaStream_t stream) {
  if (skip < 0 || g0 < 0) return SSEQS_ERR_ARG;
  SwArgs a{query_idx, query_len, good_idx, g0, n_targets, ascii, delim, skip, out, gap_a, gap_b};
  return run(affine != 0, a, stream);
}

extern "C" int sseqs_sw_scan_both(const uint8_t* query_idx, int query_len,
                                  const int32_t* good_idx, int32_t g0, int64_t n_targets,
                                  const uint8_t* ascii, const int32_t* delim, int affine_skip,
                                  int32_t* out_linear, int32_t* out_affine, int gap,
                                  int gap_open, int gap_extend, cudaStream_t stream) {
  if (g0 < 0 || n_targets < 0 || (affine_skip != 0 && affine_skip != 1)) return SSEQS_ERR_ARG;
  if (n_targets == 0) return SSEQS_OK;
  if (!out_linear || !out_affine || !delim || !ascii) return SSEQS_ERR_ARG;
  if (query_len < 0) return SSEQS_ERR_ARG;
  if (query_len > kMaxQuery) return SSEQS_ERR_UNSUPPORTED;
  if (query_len == 0) {   // as the two scans: every result -1 (sseqs/sw.cu:73, :201)
    const int grid = (int)std::min<int64_t>((n_targets + 255) / 256, 4096);
    { fill_kernel<<<grid, 256, 0, stream>>>(out_linear, n_targets, -1); count_launches(1); }
    { fill_kernel<<<grid, 256, 0, stream>>>(out_affine, n_targets, -1); count_launches(1); }
    return status_of(cudaGetLastError());
  }
  if (!query_idx) return SSEQS_ERR_ARG;
  if (!fast_domain(false, gap, 0) || !fast_domain(true, gap_open, gap_extend))
    return SSEQS_ERR_UNSUPPORTED;
  SwArgs a{query_idx, query_len, good_idx, g0, n_targets, ascii, delim, 0, out_linear, gap,
           gap_open};
  if ((query_len + 31) / 32 > kMaxFusedTpt) {   // no fused kernel: the two scans in turn
    const int st = launch_stream(a, kLin, nullptr, stream);
    if (st != SSEQS_OK) return st;
    SwArgs b = a;
    b.skip = affine_skip;
    b.out = out_affine;
    b.p0 = gap_open;
    b.p1 = gap_extend;
    return launch_stream(b, kAff, nullptr, stream);
  }
  a.p2 = gap_extend;
  a.out2 = out_affine;
  a.skip2 = affine_skip;
  return launch_stream(a, kBoth, nullptr, stream);
}

extern "C" int sseqs_sw_scan_queries(int affine, int n_queries, int tpt, const uint8_t* queries,
                                     int64_t query_stride, const int32_t* query_lens,
                                     const int32_t* good_idx, int64_t idx_stride, int32_t g0,
                                     int64_t n_targets,
                                     const uint8_t* ascii, const int32_t* delim, int skip,
                                     int32_t* out, int64_t out_stride, int gap_a, int gap_b,
                                     uint32_t* tickets, cudaStream_t stream) {
  if (n_queries < 0 || skip < 0 || g0 < 0 || n_targets < 0 || idx_stride < 0)
    return SSEQS_ERR_ARG;
  if (good_idx && idx_stride > 0 && idx_stride < n_targets) return SSEQS_ERR_ARG;
  if (n_queries == 0 || n_targets == 0) return SSEQS_OK;
  if (!queries || !query_lens || !tickets || !out || !ascii || !delim ||
      out_stride < n_targets || query_stride < 1 || query_stride > INT32_MAX)
    return SSEQS_ERR_ARG;
  if (tpt < 1 || tpt > kMaxQuery / 32) return SSEQS_ERR_UNSUPPORTED;
  const bool aff = affine != 0;
  if (!fast_domain(aff, gap_a, gap_b)) return SSEQS_ERR_UNSUPPORTED;
  // affine queries that share their targets are scored two per launch row
  // (the query-pair kernel); per-query target lists keep one query per row
  bool pair;
  {
    std::lock_guard<std::mutex> lk(cache().mu);
    pair = cache().pairing[tpt - 1];
  }
  pair = pair && aff && n_queries >= 2 && (!good_idx || idx_stride == 0);
  // launches of up to kMaxLaunchQueries queries; with pairing, an odd
  // query left over at the end runs in a one-query-per-row launch (a pair
  // row with an empty half would cost as much as a full one)
  auto launch = [&](int q0, int nq, int mode) {
    QueryTable qt{};
    qt.n = nq;
    qt.lens = query_lens + q0;
    qt.q_stride = (int32_t)query_stride;
    qt.out_stride = out_stride;
    qt.idx_stride = good_idx ? idx_stride : 0;
    const int32_t* idx0 = good_idx ? good_idx + q0 * qt.idx_stride : nullptr;
    SwArgs a{queries + (size_t)q0 * query_stride, tpt * 32, idx0, g0, n_targets,
             ascii, delim, skip, out + q0 * out_stride, gap_a, gap_b, tickets + q0};
    return launch_stream(a, mode, &qt, stream);
  };
  const int n_paired = pair ? (n_queries & ~1) : 0;
  for (int q0 = 0; q0 < n_paired; q0 += kMaxLaunchQueries) {
    const int st = launch(q0, std::min(kMaxLaunchQueries, n_paired - q0), kPair);
    if (st != SSEQS_OK) return st;
  }
  for (int q0 = n_paired; q0 < n_queries; q0 += kMaxLaunchQueries) {
    const int st = launch(q0, std::min(kMaxLaunchQueries, n_queries - q0), aff ? kAff : kLin);
    if (st != SSEQS_OK) return st;
  }
  return SSEQS_OK;
}

extern "C" int sseqs_sw_set_query_pairing(int tpt, int on) {
  if ((on != 0 && on != 1) || tpt < 0 || tpt > 64) return SSEQS_ERR_ARG;
  std::lock_guard<std::mutex> lk(cache().mu);
  for (int t = 1; t <= 64; ++t)
    if (tpt == 0 || t == tpt) cache().pairing[t - 1] = on != 0;
  return SSEQS_OK;
}

extern "C" int sseqs_sw_get_query_pairing(int tpt) {
  if (tpt < 1 || tpt > 64) return -1;
  std::lock_guard<std::mutex> lk(cache().mu);
  return cache().pairing[tpt - 1] ? 1 : 0;
}

extern "C" int sseqs_dpx_peak(uint32_t* sink, double* lane_ops_per_s, cudaStream_t stream) {
  if (!lane_ops_per_s || !sink) return SSEQS_ERR_ARG;
  return time_peak(dpx_peak_kernel, sink, lane_ops_per_s, stream);
}

extern "C" int sseqs_int16x2_peak(uint32_t* sink, double* lane_ops_per_s, cudaStream_t stream) {
  if (!lane_ops_per_s || !sink) return SSEQS_ERR_ARG;
  return time_peak(int16x2_peak_kernel, sink, lane_ops_per_s, stream);
}

extern "C" int sseqs_sw_set_variant(int affine, int tpt, int wide) {
  if (tpt < 1 || tpt > 64 || (wide != 0 && wide != 1) || affine < 0 || affine >= kModes)
    return SSEQS_ERR_ARG;
  std::lock_guard<std::mutex> lk(cache().mu);
  cache().variant[affine][tpt - 1] = wide;
  return SSEQS_OK;
}

extern "C" int sseqs_sw_get_variant(int affine, int tpt) {
  if (tpt < 1 || tpt > 64 || affine < 0 || affine >= kModes) return -1;
  std::lock_guard<std::mutex> lk(cache().mu);
  return cache().variant[affine][tpt - 1];
}

extern "C" int sseqs_sw_variant_words(int affine, int tpt, int wide) {
  if (tpt < 1 || tpt > 64 || (wide != 0 && wide != 1) || affine < 0 || affine >= kModes) return -1;
  return tables().k[0][wide][affine][tpt - 1].words;
}
