// Gapless low-rank correlation prefilter: the quantity of sseqs/fft.cu:17-415
// with sseqs/filter.cu:92-159, computed directly instead of by FFT.
//
// For a query q (Lq residues), rank-k look-up tables A (query side) and B
// (database side), a segment t (Lt <= N bytes) and N a power of two:
//   a_r[i] = A_r[pos(q[Lq-1-i])] (i < Lq),   b_r[i] = B_r[pos(t[i])] (i < Lt),
//   y      = sum_r a_r (*) b_r                (cyclic convolution of length N)
//   score  = fp16( 0.5 * max over even s of y[s] )
// pos() maps ARNDCQEGHILKMFPSTWYV to 0..19, X - * to 20 and any other byte to
// 21; B_r[21] is B_{r+1}[0] (the reference reads one entry past the row,
// sseqs/fft.cu:91,124) and 0 for the last rank.
//
// Direct form.  With j = Lq-1-i the forward query position, the linear
// correlation c[m] = sum_i a[i] b[m-i] is the sum of P(j, t[p]) along the
// diagonal p - j = m - (Lq-1) of the Lq x Lt matrix, where
//   P(j, c) = sum_r A_r[pos(q[j])] * B_r[c]
// is a per-query profile; and the cyclic y folds c once: y[s] = c[s] +
// c[s+N] (c has Lq+Lt-1 <= 2N entries), with y[s] = 0 for lags that no
// diagonal reaches.  So every score is a set of fp32 diagonal sums: one add
// per (query, target) cell, about Lq*Lt/2 useful ones per segment, instead of
// k+1 transforms of length N (N is set by the longest segment of the batch).
//
// B200 mapping: one warp per segment, lane l holding C = ceil(Lq/32)
// consecutive query columns (the query is left-padded to 32C columns with
// zero profile entries), D(j) the running sum of the diagonal ending at
// (row, j).  A row is D(j) <- D(j-1) + P(j, t[row]): a shift by one column
// (one shuffle crosses the lane boundary) and C adds.  Reading the profile
// is what bounds the kernel (shared-memory bandwidth: a profile entry per
// cell), so it is stored as fp16 -- half the bytes -- and each add takes the
// fp16 entry and the fp32 running sum in one instruction (add.f32.f16; the
// sums stay fp32).  The profile sits in shared memory, 32C entries per class,
// each lane's columns padded to an odd number of 16-byte units so the
// 128-bit loads of a warp do not conflict.  The value leaving the last column at row s is c[s]; it enters
// the maximum at once unless its partner c[s+N] exists, in which case it is
// parked in a per-warp shared array until the segment's last row, when the
// remaining diagonals (m >= Lt) are read off every column.
//
// Tensor-core form (rank k <= 4, N <= 2048; the reference's default rank is 4).
// Only even lags enter the score, so with lags m = 32u + 2v (row u, column
// v < 16) and target positions p = kk + 2v,
//   c[32u + 2v] = sum_r sum_kk a_r[32u - kk] * b_r[kk + 2v],
// a matrix product C[u, v] = sum_kk A[u, kk] B[kk, v] with
//   A[u, kk] = a_r[32u - kk]   (the query factors read backwards: a row is 16
//                                contiguous fp16 of the reversed query, rows
//                                32 elements apart -- one shared copy per CTA,
//                                loaded by ldmatrix at any (u, kk) offset),
//   B[kk, v] = b_r[kk + 2v]    (the segment's factors: a fragment register is
//                                one aligned half2 of the target array),
// and the k ranks summed into the same accumulators.  mma.sync m16n8k16
// (fp16 in, fp32 accumulate): a warp per segment, 16-row tiles of 512 lags,
// K blocks of 16 target positions that meet the tile's non-zero band only,
// two 8-column halves per A fragment.  The even-lag sums go to a per-warp
// shared array, folded there (y[s] = c[s] + c[s+N]) into the maximum.  Work
// is about (Lq + Lt) * Lt / 2 multiply-adds per rank against Lq * Lt / 2
// useful ones; the factors are rounded to fp16 (the direct form rounds the
// profile), sums stay fp32.
#include <cuda_fp16.h>

#include <algorithm>
#include <array>
#include <utility>

#include "common.cuh"

namespace sseqs {
namespace {

constexpr int kMaxRank = 20;
constexpr int kPfClasses = 22;

__device__ __forceinline__ int pf_pos(uint8_t c) {
  const uint8_t k = ascii_class(c);
  if (k < kNumAA) return k;
  return (c == 'X' || c == '-' || c == '*') ? 20 : 21;
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
  int N;                    // cyclic length
  __half* out;              // [n]
  int len_lo, len_hi;       // tensor-core form: segments with len_lo < min(len, N) <= len_hi
};

template <int C>
struct PfShape {
  static constexpr int NV = (C + 7) / 8;                       // 128-bit loads per row
  static constexpr int LW = ((NV % 2) ? NV : NV + 1) * 8;      // fp16 entries per lane (odd x 16 B)
  static constexpr int ROW = 32 * LW;                          // entries per class
  static constexpr int WARPS = C <= 32 ? 16 : 8;
  static constexpr int PARK = 16 * C;                          // parked c[s] per warp (even s)
  static constexpr size_t smem = sizeof(__half) * (size_t)kPfClasses * ROW +
                                 sizeof(float) * (size_t)WARPS * PARK + 256;
};

// fp32 + fp16 -> fp32 in one instruction
__device__ __forceinline__ float add_f32_f16(float acc, unsigned short h) {
  float r;
  asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(r) : "h"(h), "f"(acc));
  return r;
}

template <int C>
__global__ void __launch_bounds__(32 * PfShape<C>::WARPS) prefilter_kernel(PfArgs a) {
  using S = PfShape<C>;
  constexpr int J = 32 * C;
  extern __shared__ float4 smem_pf[];
  __half* prof = reinterpret_cast<__half*>(smem_pf);               // [22][ROW]
  float* park_all = reinterpret_cast<float*>(prof + kPfClasses * S::ROW);   // [WARPS][PARK]
  uint8_t* lut = reinterpret_cast<uint8_t*>(park_all + S::WARPS * S::PARK);

  for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = (uint8_t)pf_pos((uint8_t)i);
  // profile: column j of lane l = j / C sits at l*LW + j % C; real query
  // column jr = j - (J - Lq) (left padding), its residue q[jr] = qrev[Lq-1-jr]
  const int pad = J - a.Lq;
  for (int i = threadIdx.x; i < kPfClasses * S::ROW; i += blockDim.x) {
    const int c = i / S::ROW, r = i - c * S::ROW;
    const int l = r / S::LW, v = r - l * S::LW;
    const int jr = l * C + v - pad;
    float p = 0.f;
    if (v < C && jr >= 0) {
      const int qa = a.qrev[a.Lq - 1 - jr];
      for (int rk = 0; rk < a.k; ++rk) {
        const float bv = c < 21 ? a.B[rk * 21 + c] : (rk + 1 < a.k ? a.B[(rk + 1) * 21] : 0.f);
        p = fmaf(a.A[rk * 21 + qa], bv, p);
      }
    }
    prof[i] = __float2half_rn(p);
  }
  __syncthreads();

  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float* park = park_all + wib * S::PARK;
  const uint4* myprof = reinterpret_cast<const uint4*>(prof + lane * S::LW);
  const int64_t nwarps = (int64_t)gridDim.x * S::WARPS;
  const int N = a.N, Lq = a.Lq;
  const uintptr_t au = reinterpret_cast<uintptr_t>(a.ascii);
  const uint32_t* abase = reinterpret_cast<const uint32_t*>(au & ~(uintptr_t)3);
  const int64_t aoff = (int64_t)(au & 3);

  for (int64_t s = (int64_t)blockIdx.x * S::WARPS + wib; s < a.n; s += nwarps) {
    const int len = min((int)a.lengths[s], N);
    const int64_t base = a.offsets[s];
    // lags s' <= nlim have both c[s'] and c[s'+N]
    const int nlim = Lq + len - 2 - N;
    float D[C];
#pragma unroll
    for (int k = 0; k < C; ++k) D[k] = 0.f;
    float best = -INFINITY;
    for (int i0 = 0; i0 < len; i0 += 4) {
      // four target bytes from the two aligned words that hold them (a word
      // is read only when it holds a byte of the segment)
      const int64_t ap = base + i0 + aoff;
      const int64_t wi = ap >> 2;
      const uint32_t w0 = __ldg(abase + wi);
      const uint32_t w1 = ((wi + 1) << 2) < base + len + aoff ? __ldg(abase + wi + 1) : 0u;
      const uint32_t raw = __funnelshift_r(w0, w1, (uint32_t)(ap & 3) * 8u);
      const int rows = min(4, len - i0);
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (r < rows) {
          const int cls = lut[(raw >> (8 * r)) & 0xffu];
          const uint4* pr = myprof + cls * (S::ROW / 8);
          unsigned short P[S::NV * 8];
#pragma unroll
          for (int v = 0; v < S::NV; ++v) {
            const uint4 x = pr[v];
            const uint32_t w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int h = 0; h < 4; ++h)
              asm("mov.b32 {%0, %1}, %2;" : "=h"(P[8 * v + 2 * h]), "=h"(P[8 * v + 2 * h + 1])
                  : "r"(w[h]));
          }
          float left = __shfl_up_sync(0xffffffffu, D[C - 1], 1);
          if (lane == 0) left = 0.f;
#pragma unroll
          for (int k = C - 1; k > 0; --k) D[k] = add_f32_f16(D[k - 1], P[k]);
          D[0] = add_f32_f16(left, P[0]);
          const int row = i0 + r;
          if (lane == 31 && (row & 1) == 0) {          // c[row] leaves the last column
            if (row <= nlim) park[row >> 1] = D[C - 1];
            else best = fmaxf(best, D[C - 1]);
          }
        }
      }
    }
    __syncwarp();
    // diagonals m = len + Lq - 2 - jr ending on the last row (jr <= Lq - 2)
    if (len > 0) {
#pragma unroll
      for (int k = 0; k < C; ++k) {
        const int jr = lane * C + k - (J - Lq);
        const int m = len + Lq - 2 - jr;
        if (jr >= 0 && jr <= Lq - 2 && (m & 1) == 0) {
          float v = D[k];
          if (m >= N) v += park[(m - N) >> 1];
          best = fmaxf(best, v);
        }
      }
    }
    // even lags that no diagonal reaches have y = 0 (all of them when the
    // query or the segment is empty)
    if (len == 0 || Lq == 0 || Lq + len - 1 <= N - 2) best = fmaxf(best, 0.f);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) a.out[s] = __float2half_rn(0.5f * best);
    __syncwarp();
  }
}

// ------------------------------------------------------- tensor-core form
constexpr int kMmaRank = 4;            // ranks of the tensor-core form
constexpr int kMmaPass = 4;            // 16-row tiles of 512 lags accumulated per pass
constexpr int kQPad = 496;             // zero factors around the query (tile span - 16)
constexpr int kTOff = 32;              // target factor of position p at [p + kTOff]

// Sizes for a longest cyclic length (and query, segment) MAXN.
template <int MAXN, int W>
struct PfMmaShape {
  // reversed query factors per rank (fp16), whole 128-byte lines
  static constexpr int QLEN = (MAXN + 2 * kQPad + 8 + 63) / 64 * 64;
  // target factors per rank (fp16): positions -32 .. 128 * ceil((MAXN + 48) / 128) - 1,
  // the span the fill writes (zero from len on) and the fragments read (< len + 46)
  static constexpr int TLEN = kTOff + 128 * ((MAXN + 48 + 127) / 128);
  // 16-row tiles of 512 lags covering Lq + len - 1 <= 2 MAXN - 1 lags
  static constexpr int TILES = (2 * MAXN - 1 + 511) / 512;
  static constexpr int LAGS = 256 * TILES;           // even lags per warp (fp32)
  static constexpr size_t q_bytes = sizeof(__half) * kMmaRank * QLEN;
  // the even-lag sums reuse the target factors' space once the products are done
  static constexpr size_t warp_bytes = sizeof(__half) * kMmaRank * TLEN;
  static_assert(warp_bytes >= sizeof(float) * LAGS && warp_bytes % 16 == 0, "warp space");
  static constexpr size_t smem = q_bytes + W * warp_bytes + 256 + 16 * sizeof(__half) * 22;
};

// The rows of an A fragment are 64 bytes apart, so 16-byte chunk c of a
// rank's query array is stored at chunk c ^ ((c >> 3) & 3) of its 128-byte
// line: the 8 rows an ldmatrix reads then fall in 8 different bank groups.
__device__ __forceinline__ int q_swz(int i) {
  const int c = i >> 3;
  return ((c ^ ((c >> 3) & 3)) << 3) | (i & 7);
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t (&r)[4]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(addr));
}

__device__ __forceinline__ void mma_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                          uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, "
      "{%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int MAXN, int W>
__global__ void __launch_bounds__(32 * W) prefilter_mma_kernel(PfArgs a) {
  using S = PfMmaShape<MAXN, W>;
  constexpr int kQLen = S::QLEN, kTLen = S::TLEN;
  extern __shared__ float4 smem_pf[];
  __half* qf = reinterpret_cast<__half*>(smem_pf);                     // [4][kQLen]
  uint8_t* wbase = reinterpret_cast<uint8_t*>(smem_pf) + S::q_bytes;
  uint8_t* lut = wbase + W * S::warp_bytes;                           // [256]
  __half* bx = reinterpret_cast<__half*>(lut + 256);                  // [4][22] (pad 16)
  const int Lq = a.Lq, N = a.N, K = a.k;
  // reversed query factors: ar_r[x] = a_r[-x] = A_r[qrev[-x]] for -(Lq-1) <= x <= 0,
  // stored at [x + xoff]; xoff is a multiple of 8 so every ldmatrix row is aligned
  const int xoff = (Lq - 1 + kQPad + 7) & ~7;
  for (int i = threadIdx.x; i < kMmaRank * kQLen; i += blockDim.x) {
    const int r = i / kQLen, li = i - r * kQLen, x = li - xoff;
    float v = 0.f;
    if (r < K && x <= 0 && x > -Lq) v = a.A[r * 21 + a.qrev[-x]];
    qf[r * kQLen + q_swz(li)] = __float2half_rn(v);
  }
  for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = (uint8_t)pf_pos((uint8_t)i);
  for (int i = threadIdx.x; i < kMmaRank * 22; i += blockDim.x) {
    const int r = i / 22, c = i - r * 22;
    float v = 0.f;
    if (r < K) v = c < 21 ? a.B[r * 21 + c] : (r + 1 < K ? a.B[(r + 1) * 21] : 0.f);
    bx[i] = __float2half_rn(v);
  }
  __syncthreads();

  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  __half* tf = reinterpret_cast<__half*>(wbase + wib * S::warp_bytes);     // [4][kTLen]
  float* lagbuf = reinterpret_cast<float*>(tf);                              // [S::LAGS]
  const uintptr_t au = reinterpret_cast<uintptr_t>(a.ascii);
  const uint32_t* abase = reinterpret_cast<const uint32_t*>(au & ~(uintptr_t)3);
  const int64_t aoff = (int64_t)(au & 3);
  const uint32_t qf_s = (uint32_t)__cvta_generic_to_shared(qf);
  // ldmatrix x4: lane supplies row (lane & 7) + 8 * ((lane >> 3) & 1) of
  // column block 8 * (lane >> 4)
  const int lrow = (lane & 7) + 8 * ((lane >> 3) & 1), lcol = 8 * (lane >> 4);
  const int g = lane >> 2, tq = lane & 3;
  const int64_t nwarps = (int64_t)gridDim.x * W;

  for (int64_t s = (int64_t)blockIdx.x * W + wib; s < a.n; s += nwarps) {
    const int len = min((int)a.lengths[s], N);
    if (len <= a.len_lo || len > a.len_hi) continue;     // another launch scores it
    // positions -32 .. -1 are zero (the lag sums of the previous segment
    // shared this space)
    for (int i = lane; i < kMmaRank * (kTOff / 2); i += 32)
      reinterpret_cast<__half2*>(tf + (i / (kTOff / 2)) * kTLen)[i % (kTOff / 2)] =
          __float2half2_rn(0.f);
    // target factors b_r[p] for p in [0, len + 48), zero from len on: lane l
    // takes positions 4(l + 32m) .. +3, from the aligned words w and w + 1
    // that hold them (w from this lane, w + 1 from the next one); all loads of
    // the segment are issued before any is used, and a word is read only when
    // it holds a byte of the segment
    {
      constexpr int kM = (MAXN + 48 + 127) / 128;
      const int64_t ap = a.offsets[s] + aoff;
      const int64_t w0 = ap >> 2;
      const int64_t wend = (ap + len + 3) >> 2;          // words holding segment bytes
      const uint32_t sh = (uint32_t)(ap & 3) * 8u;
      const int nm = (len + 48 + 127) / 128;
      uint32_t w[kM + 1];
#pragma unroll
      for (int m = 0; m <= kM; ++m) {
        const int64_t wi = w0 + lane + 32 * m;
        w[m] = (m <= nm && wi < wend) ? __ldg(abase + wi) : 0u;
      }
#pragma unroll
      for (int m = 0; m < kM; ++m) {
        if (m < nm) {
          uint32_t nx = __shfl_down_sync(0xffffffffu, w[m], 1);
          const uint32_t wrap = __shfl_sync(0xffffffffu, w[m + 1], 0);
          if (lane == 31) nx = wrap;
          const uint32_t raw = __funnelshift_r(w[m], nx, sh);
          const int p0 = 4 * (lane + 32 * m);
          int c[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) c[i] = p0 + i < len ? lut[(raw >> (8 * i)) & 0xffu] : -1;
#pragma unroll
          for (int r = 0; r < kMmaRank; ++r) {
            __half h[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) h[i] = c[i] >= 0 ? bx[r * 22 + c[i]] : __float2half_rn(0.f);
            __half2* dst = reinterpret_cast<__half2*>(tf + r * kTLen + kTOff + p0);
            dst[0] = __halves2half2(h[0], h[1]);
            dst[1] = __halves2half2(h[2], h[3]);
          }
        }
      }
    }
    __syncwarp();
    // lags 0 .. Lq + len - 2 in rows u = lag / 32, tiles of 16 rows, kMmaPass
    // tiles per pass; each pass's sums stay in registers until the last pass
    // is done, then go to lagbuf[16u + v] (even lag 32u + 2v), over the
    // target factors
    const int rows = (Lq + len - 1 + 31) / 32;
    const int ntiles = (rows + 15) / 16;
    float sums[S::TILES][2][4];
#pragma unroll
    for (int P = 0; P < S::TILES / kMmaPass; ++P) {
      const int t0 = P * kMmaPass;
      if (t0 < ntiles) {
        // two accumulator sets (even and odd ranks) halve the chains of
        // dependent MMAs
        float acc[kMmaPass][2][2][4];
#pragma unroll
        for (int tj = 0; tj < kMmaPass; ++tj)
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[tj][0][h][e] = acc[tj][1][h][e] = 0.f;
        if (len > 0) {
          // kk ranges over [-30, len); tile ti needs kk in (512 ti - Lq, 512 ti + 480]
          const int kb_lo = max(-32, ((512 * t0 - Lq - 14) >> 4) << 4);
          const int kb_hi = min(len - 1, 512 * (t0 + kMmaPass - 1) + 480);
          for (int kb = kb_lo; kb <= kb_hi; kb += 16) {
            uint32_t bf[kMmaRank][2][2];
#pragma unroll
            for (int r = 0; r < kMmaRank; ++r) {
              const uint32_t* tr =
                  reinterpret_cast<const uint32_t*>(tf + r * kTLen + kTOff + kb);
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const int v = g + 8 * h;             // column: lag 32u + 2v
                bf[r][h][0] = tr[tq + v];           // b[kb + 2tq + 2v .. +1]
                bf[r][h][1] = tr[tq + v + 4];       // b[kb + 8 + 2tq + 2v .. +1]
              }
            }
#pragma unroll
            for (int tj = 0; tj < kMmaPass; ++tj) {
              const int ti = t0 + tj;
              if (ti < ntiles && kb + 15 > 512 * ti - Lq && kb <= 512 * ti + 480) {
                // row u = 16 ti + lrow, columns kb + lcol .. +7: ar[kb + lcol - 32u ...]
                const uint32_t qa =
                    qf_s + 2u * (uint32_t)q_swz(kb + lcol - 32 * (16 * ti + lrow) + xoff);
                uint32_t af[kMmaRank][4];
#pragma unroll
                for (int r = 0; r < kMmaRank; ++r)
                  if (r < K) ldsm_x4(qa + (uint32_t)(2 * r * kQLen), af[r]);
#pragma unroll
                for (int r = 0; r < kMmaRank; ++r) {
                  if (r < K) {
                    mma_16816(acc[tj][r & 1][0], af[r], bf[r][0][0], bf[r][0][1]);
                    mma_16816(acc[tj][r & 1][1], af[r], bf[r][1][0], bf[r][1][1]);
                  }
                }
              }
            }
          }
        }
#pragma unroll
        for (int tj = 0; tj < kMmaPass; ++tj)
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int e = 0; e < 4; ++e) sums[t0 + tj][h][e] = acc[tj][0][h][e] + acc[tj][1][h][e];
      }
    }
    __syncwarp();                                // every lane's factor reads are done
#pragma unroll
    for (int ti = 0; ti < S::TILES; ++ti) {
      if (ti < ntiles) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int u = 16 * ti + g + 8 * (e >> 1);
            const int v = 2 * tq + (e & 1) + 8 * h;
            lagbuf[16 * u + v] = sums[ti][h][e];
          }
        }
      }
    }
    __syncwarp();
    // y[s] = c[s] + c[s + N] over even s < N; lags past the computed tiles
    // are 0, and so are lags no diagonal reaches
    const int lim = 256 * ntiles;
    float best = -INFINITY;
    for (int e1 = lane; e1 < N / 2; e1 += 32) {
      const int e2 = e1 + N / 2;
      const float y = (e1 < lim ? lagbuf[e1] : 0.f) + (e2 < lim ? lagbuf[e2] : 0.f);
      best = fmaxf(best, y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) a.out[s] = __float2half_rn(0.5f * best);
    __syncwarp();
  }
}

template <int MAXN, int W>
int launch_pf_mma(const PfArgs& a, cudaStream_t stream) {
  using S = PfMmaShape<MAXN, W>;
  static_assert(S::TILES % kMmaPass == 0, "whole passes");
  const void* fn = (const void*)prefilter_mma_kernel<MAXN, W>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem) !=
      cudaSuccess)
    return SSEQS_ERR_CUDA;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, 32 * W, S::smem) != cudaSuccess ||
      nb < 1)
    return SSEQS_ERR_CUDA;
  const int64_t need = (a.n + W - 1) / W;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)device_sm_count() * nb));
  { prefilter_mma_kernel<MAXN, W><<<grid, 32 * W, S::smem, stream>>>(a); count_launches(1); }
  return status_of(cudaGetLastError());
}

// ------------------------------------------------------------ dispatch
using PfFn = void (*)(PfArgs);
struct PfInfo {
  PfFn fn;
  size_t smem;
  int threads;
};

template <int... I>
std::array<PfInfo, sizeof...(I)> pf_table(std::integer_sequence<int, I...>) {
  return {{PfInfo{prefilter_kernel<I + 1>, PfShape<I + 1>::smem, 32 * PfShape<I + 1>::WARPS}...}};
}

int launch_pf(const PfArgs& a, cudaStream_t stream) {
  // tensor-core form for ranks up to 4: segments and queries up to 1024
  // residues with 16 warps per CTA; longer ones (cyclic length 2048) with the
  // bigger buffers of the 2048 form, 8 warps per CTA
  if (a.k <= kMmaRank && a.Lq >= 1 && a.N <= 2048) {
    if (a.Lq <= 1024) {
      PfArgs b = a;
      b.len_lo = -1;
      b.len_hi = 1024;
      const int st = launch_pf_mma<1024, 16>(b, stream);
      if (st != SSEQS_OK || a.N <= 1024) return st;
      b.len_lo = 1024;
      b.len_hi = a.N;
      return launch_pf_mma<2048, 8>(b, stream);
    }
    PfArgs b = a;
    b.len_lo = -1;
    b.len_hi = a.N;
    return launch_pf_mma<2048, 8>(b, stream);
  }
  static const auto table = pf_table(std::make_integer_sequence<int, 64>{});
  const int C = std::max(1, (a.Lq + 31) / 32);
  const PfInfo& info = table[C - 1];
  if (cudaFuncSetAttribute((const void*)info.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)info.smem) != cudaSuccess)
    return SSEQS_ERR_CUDA;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)info.fn, info.threads,
                                                    info.smem) != cudaSuccess || nb < 1)
    return SSEQS_ERR_CUDA;
  const int warps = info.threads / 32;
  const int64_t need = (a.n + warps - 1) / warps;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)device_sm_count() * nb));
  { info.fn<<<grid, info.threads, info.smem, stream>>>(a); count_launches(1); }
  return status_of(cudaGetLastError());
}

}  // namespace
}  // namespace sseqs

using namespace sseqs;

extern "C" size_t sseqs_prefilter_workspace_bytes(int n, int k) {
  if (n < 2 || k < 1) return 0;
  return 256;
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
  if (n_segments == 0) return SSEQS_OK;
  PfArgs a{ascii, offsets, lengths, n_segments, lut_a, lut_b, query_pos_reversed, query_len, k, n,
           reinterpret_cast<__half*>(out_scores), -1, n};
  return launch_pf(a, stream);
}
