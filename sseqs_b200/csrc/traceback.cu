// Affine local alignment with traceback (replaces the Triton kernels
// sseqs/sw.py:408-563 and :569-768 driven by sseqs/sw.py:27-219).
//
// Recurrence (textbook Gotoh, gaps open from H), i = query, j = target:
//   M(i,j)  = s(q_i, t_j) + H(i-1,j-1)
//   Ix(i,j) = max(H(i-1,j) - open, Ix(i-1,j) - ext)     Ix(0,j) := -16384
//   Iy(i,j) = max(H(i,j-1) - open, Iy(i,j-1) - ext)     Iy(i,0) := -16384
//   H(i,j)  = max(0, M, Ix, Iy),  H = 0 on row 0 and column 0,
// s = BLOSUM62 for two upper-case standard residues, else -5.  The end cell
// is the first cell in query-major order whose H equals the best score; the
// walk back takes, at every cell, the first state equal to H in the order M,
// Ix, Iy (diagonal, up, left) and stops at H == 0 or a border.  At every
// cell that state's own back-pointer condition holds by construction (M is
// s + H(i-1,j-1); Ix and Iy are the max of their two sources), so a 2-bit
// code per cell (stop / diag / up / left) carries the whole walk.
//
// B200 mapping: one warp per target.  The query is processed in blocks of
// 32 rows (one row per lane); the block sweeps the target as a wavefront,
// lane l computing column s-l at step s and receiving H/Ix of the row above
// from lane l-1 by shuffle.  Lane 0 reads the previous block's last row from
// a per-target buffer that lane 31 rewrites in place.  Codes are packed 16
// per word into the workspace; the walk then reads them from L2.
#include <algorithm>

#include "common.cuh"

namespace sseqs {
namespace {

constexpr int kNegBorder = -16384;

struct TbArgs {
  const uint8_t* q;
  int Lq;
  const uint8_t* tbytes;
  const int64_t* toff;
  const int32_t* tlen;
  int B;
  int go, ge;
  uint32_t* dir;            // workspace: codes, dir_stride words per target
  int64_t dir_stride;
  int32_t* top;             // workspace: previous block's last row, top_stride ints per target
  int64_t top_stride;
  int32_t* best;            // [B]
  int32_t* info;            // [B][5]: alen, q_start, q_end, t_start, t_end
  uint8_t* q_al;            // [B][cap], filled from the end
  uint8_t* t_al;
  int cap;
  int32_t* mfull;           // optional [B][Lq+1][tcols]
  int tcols;
  int tmax;                 // longest target the workspace was sized for
};

__device__ __forceinline__ int tb_class(uint8_t c) {
  return ascii_class(c) < kNumAA ? (int)ascii_class(c) : -1;
}

__global__ void __launch_bounds__(32) traceback_kernel(TbArgs a) {
  __shared__ int8_t sb62[400];
  __shared__ int8_t scls[256];
  for (int i = threadIdx.x; i < 400; i += 32) sb62[i] = blosum62(i / 20, i % 20);
  for (int i = threadIdx.x; i < 256; i += 32) scls[i] = (int8_t)tb_class((uint8_t)i);
  __syncwarp();

  const int b = blockIdx.x;
  if (b >= a.B) return;
  const int lane = threadIdx.x;
  const int Lq = a.Lq;
  const int Lt = a.tlen[b];
  if (Lt < 0 || Lt > a.tmax) {   // outside the workspace the caller sized
    if (lane == 0) {
      a.best[b] = -1;
      for (int k = 0; k < 5; ++k) a.info[(int64_t)b * 5 + k] = -1;
    }
    return;
  }
  const uint8_t* t = a.tbytes + a.toff[b];
  const int W16 = (Lt + 15) >> 4;
  uint32_t* dir = a.dir + (int64_t)b * a.dir_stride;
  int32_t* topH = a.top + (int64_t)b * a.top_stride;
  int32_t* topX = topH + (Lt + 1);
  int32_t* mf = a.mfull ? a.mfull + (int64_t)b * (Lq + 1) * a.tcols : nullptr;

  for (int j = lane; j <= Lt; j += 32) { topH[j] = 0; topX[j] = kNegBorder; }
  __syncwarp();

  int bestv = 0, bi = 0x7fffffff, bj = 0x7fffffff;
  if (Lq > 0 && Lt > 0) {
    for (int rb = 0; rb < Lq; rb += 32) {
      const int i = rb + lane + 1;                 // this lane's row (1-based)
      const bool row_ok = i <= Lq;
      const int qc = row_ok ? scls[a.q[i - 1]] : -1;
      int hleft = 0, yleft = kNegBorder;           // H(i,j-1), Iy(i,j-1)
      int hdiag = 0;                               // H(i-1,j-1)
      int hup_in = 0, xup_in = kNegBorder;         // from lane-1, previous step
      uint32_t codes = 0;
      const int steps = Lt + 31;
      for (int s = 0; s < steps; ++s) {
        const int j = s - lane + 1;                // this lane's column (1-based)
        // values of the row above for column j
        int hup = __shfl_up_sync(0xffffffffu, hup_in, 1);
        int xup = __shfl_up_sync(0xffffffffu, xup_in, 1);
        if (lane == 0 && j >= 1 && j <= Lt) { hup = topH[j]; xup = topX[j]; }
        const bool live = row_ok && j >= 1 && j <= Lt;
        int h = 0, x = kNegBorder;
        if (live) {
          const int tc = scls[__ldg(t + j - 1)];
          const int sc = (qc >= 0 && tc >= 0) ? sb62[qc * 20 + tc] : -5;
          const int hd = (j == 1) ? 0 : hdiag;
          const int m = sc + hd;
          const int xsrc = (i == 1) ? kNegBorder : xup;
          x = max(hup - a.go, xsrc - a.ge);
          const int ysrc = (j == 1) ? kNegBorder : yleft;
          const int y = max(hleft - a.go, ysrc - a.ge);
          h = max(max(0, m), max(x, y));
          const uint32_t code = h == 0 ? 0u : (h == m ? 1u : (h == x ? 2u : 3u));
          codes |= code << (((j - 1) & 15) * 2);
          if (((j & 15) == 0) || j == Lt) {
            dir[(int64_t)(i - 1) * W16 + ((j - 1) >> 4)] = codes;
            codes = 0;
          }
          if (h > bestv || (h == bestv && h > 0 && (i < bi || (i == bi && j < bj)))) {
            bestv = h; bi = i; bj = j;
          }
          if (mf) mf[(int64_t)i * a.tcols + j] = m;
          hleft = h;
          yleft = y;
        }
        if (lane == 31 && live) { topH[j] = h; topX[j] = x; }
        // next step: this lane's diagonal is the value just received from above
        hdiag = hup;
        hup_in = h;
        xup_in = x;
        __syncwarp();
      }
      __syncwarp();
    }
  }
  // warp reduction: best value, then the first cell in query-major order
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int ov = __shfl_xor_sync(0xffffffffu, bestv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    const int oj = __shfl_xor_sync(0xffffffffu, bj, o);
    if (ov > bestv || (ov == bestv && (oi < bi || (oi == bi && oj < bj)))) {
      bestv = ov; bi = oi; bj = oj;
    }
  }
  if (lane != 0) return;
  a.best[b] = bestv;
  int32_t* inf = a.info + (int64_t)b * 5;
  inf[0] = 0; inf[1] = -1; inf[2] = -1; inf[3] = -1; inf[4] = -1;
  if (!(bestv > 0 && Lq > 0 && Lt > 0)) return;
  uint8_t* qa = a.q_al + (int64_t)b * a.cap;
  uint8_t* ta = a.t_al + (int64_t)b * a.cap;
  int ci = bi, cj = bj, n = 0;
  for (int it = 0; it < Lq + Lt + 2; ++it) {
    if (ci <= 0 || cj <= 0) break;
    const uint32_t w = dir[(int64_t)(ci - 1) * W16 + ((cj - 1) >> 4)];
    const uint32_t code = (w >> (((cj - 1) & 15) * 2)) & 3u;
    if (code == 0) break;
    const int pos = a.cap - 1 - n;
    if (code == 1) { qa[pos] = a.q[ci - 1]; ta[pos] = t[cj - 1]; --ci; --cj; }
    else if (code == 2) { qa[pos] = a.q[ci - 1]; ta[pos] = '-'; --ci; }
    else { qa[pos] = '-'; ta[pos] = t[cj - 1]; --cj; }
    ++n;
  }
  if (n > 0) {
    inf[0] = n; inf[1] = ci; inf[2] = bi - 1; inf[3] = cj; inf[4] = bj - 1;
  }
}

}  // namespace
}  // namespace sseqs

using namespace sseqs;

namespace {
inline int64_t dir_words(int query_len, int tmax) { return (int64_t)query_len * ((tmax + 15) / 16); }
inline int64_t top_ints(int tmax) { return 2 * (int64_t)(tmax + 1); }
}  // namespace

extern "C" size_t sseqs_backtrack_workspace_bytes(int query_len, int max_target_len, int B) {
  if (B < 0 || query_len < 0 || max_target_len < 0) return 0;
  return (size_t)B * 4 * (size_t)(dir_words(query_len, max_target_len) + top_ints(max_target_len)) + 256;
}

extern "C" int sseqs_backtrack_affine(const uint8_t* query, int query_len, const uint8_t* tbytes,
                                      const int64_t* toff, const int32_t* tlen, int max_target_len,
                                      int B, int gap_open, int gap_extend, int32_t* best,
                                      int32_t* info, uint8_t* q_aligned, uint8_t* t_aligned,
                                      int cap, int32_t* m_full, int tcols, void* workspace,
                                      size_t ws_bytes, cudaStream_t stream) {
  if (B < 0 || query_len < 0 || max_target_len < 0) return SSEQS_ERR_ARG;
  if (B == 0) return SSEQS_OK;
  if (!tbytes || !toff || !tlen || !best || !info || !q_aligned || !t_aligned ||
      (query_len > 0 && !query))
    return SSEQS_ERR_ARG;
  if (cap < query_len + max_target_len) return SSEQS_ERR_ARG;
  if (m_full && tcols < max_target_len + 1) return SSEQS_ERR_ARG;
  if (!workspace || ws_bytes < sseqs_backtrack_workspace_bytes(query_len, max_target_len, B))
    return SSEQS_ERR_WORKSPACE;
  uint32_t* dir = reinterpret_cast<uint32_t*>(workspace);
  const int64_t ds = dir_words(query_len, max_target_len);
  int32_t* top = reinterpret_cast<int32_t*>(dir + (int64_t)B * ds);
  TbArgs a{query, query_len, tbytes, toff, tlen, B, gap_open, gap_extend, dir, ds,
           top, top_ints(max_target_len), best, info, q_aligned, t_aligned, cap, m_full, tcols,
           max_target_len};
  { traceback_kernel<<<B, 32, 0, stream>>>(a); count_launches(1); }
  return status_of(cudaGetLastError());
}
