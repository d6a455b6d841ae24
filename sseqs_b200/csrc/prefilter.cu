// Gapless low-rank correlation prefilter (the quantity of sseqs/fft.cu:17-415
// with sseqs/filter.cu:92-159).
//
// For a query q, rank-k look-up tables A (query side) and B (database side)
// and a segment t, with N a power of two and H = N/2:
//   a_r[i] = A_r[pos(q[Lq-1-i])] (i < Lq),   b_r[i] = B_r[pos(t[i])] (i < Lt),
//   y      = sum_r a_r (*) b_r                (cyclic convolution of length N)
//   score  = fp16( 0.5 * max_n y[2n] )        (even lags only)
// pos() maps ARNDCQEGHILKMFPSTWYV to 0..19, X - * to 20 and any other byte to
// 21; B_r[21] is B_{r+1}[0] (the reference reads one entry past the row,
// sseqs/fft.cu:91,124) and 0 for the last rank.
//
// B200 mapping: one warp per segment, fp32.  Real inputs of length N are
// packed as z[n] = x[2n] + i x[2n+1] and transformed by a 32-lane radix-2
// FFT of length H (H/32 complex values per lane; stages whose butterfly
// partner lives in another lane exchange through __shfl_xor_sync).  The
// forward transform is decimation-in-time on bit-reversed input (natural
// order out), the rank products are summed in the frequency domain
// (P = sum_r Q_r X_r), and a single decimation-in-frequency inverse follows
// -- its output order does not matter because only the maximum is kept.
// The query spectra Q_r are computed once per (query, N) by the same code.
// Twiddles come from a shared table filled with sincospif.
#include <cuda_fp16.h>

#include <algorithm>

#include "common.cuh"

namespace sseqs {
namespace {

constexpr int kMaxRank = 20;
constexpr int kPfWarps = 4;

__device__ __forceinline__ int pf_pos(uint8_t c) {
  const uint8_t k = ascii_class(c);
  if (k < kNumAA) return k;
  return (c == 'X' || c == '-' || c == '*') ? 20 : 21;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 conj2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 shfl_xor2(float2 v, int m) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ float2 shfl2(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// tw[k] = exp(-2 pi i k / N), k < H
template <int LOG_H>
__device__ void fill_twiddles(float2* tw) {
  constexpr int H = 1 << LOG_H;
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    float s, c;
    sincospif(-(float)k / (float)H, &s, &c);   // -2k/N = -k/H
    tw[k] = make_float2(c, s);
  }
}

// Forward DIT of v (bit-reversed input, natural output); lane l holds
// indices l*T .. l*T+T-1.
template <int LOG_H>
__device__ __forceinline__ void fft_dit(float2 (&v)[(1 << LOG_H) / 32 > 0 ? (1 << LOG_H) / 32 : 1],
                                        const float2* tw, int lane) {
  constexpr int H = 1 << LOG_H, T = H / 32, N = 2 * H;
  const int base = lane * T;
#pragma unroll
  for (int s = 0; s < LOG_H; ++s) {
    const int half = 1 << s;
    const int step = N / (2 * half);        // W_m^j = tw[j * N/m]
    if (half < T) {
#pragma unroll
      for (int i = 0; i < T; ++i) {
        const int g = base + i;
        if ((g & half) == 0) {
          const float2 w = tw[(g & (half - 1)) * step];
          const float2 a = v[i], t = cmul(v[i ^ half], w);
          v[i] = cadd(a, t);
          v[i ^ half] = csub(a, t);
        }
      }
    } else {
      const int ld = half / T;
#pragma unroll
      for (int i = 0; i < T; ++i) {
        const int g = base + i;
        const float2 a = v[i], b = shfl_xor2(a, ld);
        const float2 w = tw[(g & (half - 1)) * step];
        v[i] = ((g & half) == 0) ? cadd(a, cmul(b, w)) : csub(b, cmul(a, w));
      }
    }
  }
}

// Inverse DIF (natural input, bit-reversed output), unnormalised.
template <int LOG_H>
__device__ __forceinline__ void ifft_dif(float2 (&v)[(1 << LOG_H) / 32 > 0 ? (1 << LOG_H) / 32 : 1],
                                         const float2* tw, int lane) {
  constexpr int H = 1 << LOG_H, T = H / 32, N = 2 * H;
  const int base = lane * T;
#pragma unroll
  for (int s = LOG_H - 1; s >= 0; --s) {
    const int half = 1 << s;
    const int step = N / (2 * half);
    if (half < T) {
#pragma unroll
      for (int i = 0; i < T; ++i) {
        const int g = base + i;
        if ((g & half) == 0) {
          const float2 w = conj2(tw[(g & (half - 1)) * step]);
          const float2 a = v[i], b = v[i ^ half];
          v[i] = cadd(a, b);
          v[i ^ half] = cmul(csub(a, b), w);
        }
      }
    } else {
      const int ld = half / T;
#pragma unroll
      for (int i = 0; i < T; ++i) {
        const int g = base + i;
        const float2 a = v[i], b = shfl_xor2(a, ld);
        const float2 w = conj2(tw[(g & (half - 1)) * step]);
        v[i] = ((g & half) == 0) ? cadd(a, b) : cmul(csub(b, a), w);
      }
    }
  }
}

// After fft_dit of a packed real signal: X[k] for this lane's k (written to
// X[]), and X[H] (returned; meaningful on lane 0).
template <int LOG_H>
__device__ __forceinline__ float unpack_real(float2 (&v)[(1 << LOG_H) / 32 > 0 ? (1 << LOG_H) / 32 : 1],
                                             float2 (&X)[(1 << LOG_H) / 32 > 0 ? (1 << LOG_H) / 32 : 1],
                                             const float2* tw, int lane) {
  constexpr int H = 1 << LOG_H, T = H / 32;
  float xh = 0.f;
#pragma unroll
  for (int j = 0; j < T; ++j) {
    const int k = lane * T + j;
    const int mj = (j == 0) ? 0 : T - j;
    const int ml = (j == 0) ? ((32 - lane) & 31) : 31 - lane;
    const float2 gm = shfl2(v[mj], ml);
    if (k == 0) {
      X[j] = make_float2(v[0].x + v[0].y, 0.f);
      xh = v[0].x - v[0].y;
    } else {
      const float2 S = cadd(v[j], conj2(gm)), D = csub(v[j], conj2(gm));
      const float2 WD = cmul(tw[k], D);
      X[j] = make_float2(0.5f * (S.x + WD.y), 0.5f * (S.y - WD.x));
    }
  }
  return xh;
}

struct PfArgs {
  const uint8_t* ascii;
  const int64_t* offsets;
  const int32_t* lengths;
  int64_t n;
  const float* A;           // [k][21] query side
  const float* B;           // [k][21] database side
  const uint8_t* qrev;      // query positions, reversed, already mapped (0..20)
  int Lq;
  int k;
  float2* qspec;            // [k][H+1]
  __half* out;              // [n]
};

// One warp per rank: Q_r = DFT_N(a_r), k = 0..H.
template <int LOG_H>
__global__ void __launch_bounds__(32) query_spectrum_kernel(PfArgs a) {
  constexpr int H = 1 << LOG_H, T = H / 32, N = 2 * H;
  __shared__ float2 tw[H];
  fill_twiddles<LOG_H>(tw);
  __syncwarp();
  const int r = blockIdx.x, lane = threadIdx.x;
  if (r >= a.k) return;
  float2 v[T], X[T];
#pragma unroll
  for (int j = 0; j < T; ++j) {
    const int p = (int)(__brev((unsigned)(lane * T + j)) >> (32 - LOG_H));
    const int i0 = 2 * p, i1 = 2 * p + 1;
    const float x0 = (i0 < a.Lq && i0 < N) ? a.A[r * 21 + a.qrev[i0]] : 0.f;
    const float x1 = (i1 < a.Lq && i1 < N) ? a.A[r * 21 + a.qrev[i1]] : 0.f;
    v[j] = make_float2(x0, x1);
  }
  fft_dit<LOG_H>(v, tw, lane);
  const float xh = unpack_real<LOG_H>(v, X, tw, lane);
  float2* row = a.qspec + (int64_t)r * (H + 1);
#pragma unroll
  for (int j = 0; j < T; ++j) row[lane * T + j] = X[j];
  if (lane == 0) row[H] = make_float2(xh, 0.f);
}

template <int LOG_H>
__global__ void __launch_bounds__(32 * kPfWarps) prefilter_kernel(PfArgs a) {
  constexpr int H = 1 << LOG_H, T = H / 32, N = 2 * H;
  extern __shared__ float4 smem_pf[];
  float2* tw = reinterpret_cast<float2*>(smem_pf);                 // H
  float2* Q = tw + H;                                             // k*(H+1)
  float* Bt = reinterpret_cast<float*>(Q + a.k * (H + 1));        // k*23
  uint8_t* cls_all = reinterpret_cast<uint8_t*>(Bt + a.k * 23);   // warps*N
  fill_twiddles<LOG_H>(tw);
  for (int i = threadIdx.x; i < a.k * (H + 1); i += blockDim.x) Q[i] = a.qspec[i];
  for (int i = threadIdx.x; i < a.k * 23; i += blockDim.x) {
    const int r = i / 23, c = i % 23;
    float v = 0.f;
    if (c < 21) v = a.B[r * 21 + c];
    else if (c == 21) v = (r + 1 < a.k) ? a.B[(r + 1) * 21] : 0.f;
    Bt[i] = v;                                                    // class 22: padding, 0
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint8_t* cls = cls_all + wib * N;
  const int64_t nwarps = (int64_t)gridDim.x * kPfWarps;
  for (int64_t s = (int64_t)blockIdx.x * kPfWarps + wib; s < a.n; s += nwarps) {
    const int len = min((int)a.lengths[s], N);
    const uint8_t* t = a.ascii + a.offsets[s];
    for (int i = lane; i < N; i += 32) cls[i] = i < len ? (uint8_t)pf_pos(t[i]) : (uint8_t)22;
    __syncwarp();
    float2 P[T];
    float ph = 0.f;
#pragma unroll
    for (int j = 0; j < T; ++j) P[j] = make_float2(0.f, 0.f);
    for (int r = 0; r < a.k; ++r) {
      const float* br = Bt + r * 23;
      float2 v[T];
#pragma unroll
      for (int j = 0; j < T; ++j) {
        const int p = (int)(__brev((unsigned)(lane * T + j)) >> (32 - LOG_H));
        v[j] = make_float2(br[cls[2 * p]], br[cls[2 * p + 1]]);
      }
      fft_dit<LOG_H>(v, tw, lane);
      // unpack X_r[k] (as unpack_real) and accumulate P += Q_r X_r at once;
      // v is only read here, so the mate values stay valid
      const float2* q = Q + r * (H + 1);
#pragma unroll
      for (int j = 0; j < T; ++j) {
        const int k = lane * T + j;
        const int mj = (j == 0) ? 0 : T - j;
        const int ml = (j == 0) ? ((32 - lane) & 31) : 31 - lane;
        const float2 gm = shfl2(v[mj], ml);
        float2 X;
        if (k == 0) {
          X = make_float2(v[0].x + v[0].y, 0.f);
          ph += q[H].x * (v[0].x - v[0].y);
        } else {
          const float2 S = cadd(v[j], conj2(gm)), D = csub(v[j], conj2(gm));
          const float2 WD = cmul(tw[k], D);
          X = make_float2(0.5f * (S.x + WD.y), 0.5f * (S.y - WD.x));
        }
        P[j] = cadd(P[j], cmul(q[k], X));
      }
    }
    __syncwarp();
    // pack Z[k] = DFT_H(y_even + i y_odd) from P = DFT_N(y)
    float2 Z[T];
#pragma unroll
    for (int j = 0; j < T; ++j) {
      const int k = lane * T + j;
      const int mj = (j == 0) ? 0 : T - j;
      const int ml = (j == 0) ? ((32 - lane) & 31) : 31 - lane;
      const float2 pm = shfl2(P[mj], ml);
      if (k == 0) {
        Z[j] = make_float2(0.5f * (P[0].x + ph), 0.5f * (P[0].x - ph));
      } else {
        const float2 S = cadd(P[j], conj2(pm)), D = csub(P[j], conj2(pm));
        const float2 WD = cmul(conj2(tw[k]), D);
        Z[j] = make_float2(0.5f * (S.x - WD.y), 0.5f * (S.y + WD.x));
      }
    }
    ifft_dif<LOG_H>(Z, tw, lane);
    float m = Z[0].x;
#pragma unroll
    for (int j = 1; j < T; ++j) m = fmaxf(m, Z[j].x);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) a.out[s] = __float2half_rn(m * (0.5f / (float)H));
    __syncwarp();
  }
}

template <int LOG_H>
int launch_pf(PfArgs a, cudaStream_t stream) {
  constexpr int H = 1 << LOG_H, N = 2 * H;
  { query_spectrum_kernel<LOG_H><<<a.k, 32, 0, stream>>>(a); count_launches(1); }
  if (a.n == 0) return status_of(cudaGetLastError());
  const size_t smem = sizeof(float2) * (H + (size_t)a.k * (H + 1)) + sizeof(float) * a.k * 23 +
                      (size_t)kPfWarps * N;
  if (cudaFuncSetAttribute(prefilter_kernel<LOG_H>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return SSEQS_ERR_CUDA;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, prefilter_kernel<LOG_H>, 32 * kPfWarps,
                                                    smem) != cudaSuccess || nb < 1)
    return SSEQS_ERR_CUDA;
  const int64_t need = (a.n + kPfWarps - 1) / kPfWarps;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)device_sm_count() * nb));
  { prefilter_kernel<LOG_H><<<grid, 32 * kPfWarps, smem, stream>>>(a); count_launches(1); }
  return status_of(cudaGetLastError());
}

}  // namespace
}  // namespace sseqs

using namespace sseqs;

extern "C" size_t sseqs_prefilter_workspace_bytes(int n, int k) {
  if (n < 2 || k < 1) return 0;
  return sizeof(float2) * (size_t)k * (size_t)(n / 2 + 1) + 256;
}

extern "C" int sseqs_prefilter(const uint8_t* ascii, const int64_t* offsets, const int32_t* lengths,
                               int64_t n_segments, const uint8_t* query_pos_reversed,
                               int query_len, const float* lut_a, const float* lut_b, int k,
                               int n, void* out_scores, void* workspace, size_t ws_bytes,
                               cudaStream_t stream) {
  if (n_segments < 0 || query_len < 0 || k < 1 || k > kMaxRank) return SSEQS_ERR_ARG;
  if (n < 64 || n > 2048 || (n & (n - 1)) != 0) return SSEQS_ERR_UNSUPPORTED;
  if (query_len > n) return SSEQS_ERR_ARG;
  if (!lut_a || !lut_b || (query_len > 0 && !query_pos_reversed)) return SSEQS_ERR_ARG;
  if (n_segments > 0 && (!ascii || !offsets || !lengths || !out_scores)) return SSEQS_ERR_ARG;
  if (!workspace || ws_bytes < sseqs_prefilter_workspace_bytes(n, k)) return SSEQS_ERR_WORKSPACE;
  PfArgs a{ascii, offsets, lengths, n_segments, lut_a, lut_b, query_pos_reversed, query_len, k,
           reinterpret_cast<float2*>(workspace), reinterpret_cast<__half*>(out_scores)};
  switch (n) {
    case 64: return launch_pf<5>(a, stream);
    case 128: return launch_pf<6>(a, stream);
    case 256: return launch_pf<7>(a, stream);
    case 512: return launch_pf<8>(a, stream);
    case 1024: return launch_pf<9>(a, stream);
    case 2048: return launch_pf<10>(a, stream);
  }
  return SSEQS_ERR_UNSUPPORTED;
}
