// Kernels of the learned prefilter: a 1D-conv sequence embedder (forward and
// backward in BF16 on the tensor cores, fp32 accumulation), its optimiser,
// and the FP8 database scoring GEMM with fused candidate selection.
//
// Activations of a set of sequences live in one row-major [P x C] bf16
// matrix: the sequences one after another, each followed by at least two
// zero rows, with two zero rows before the first.  A width-5 convolution
// then needs no im2col buffer: the 5 input rows p-2 .. p+2 of output row p
// are contiguous, so im2col(X) is the [P x 5C] matrix whose row p starts at
// X + (p-2)*C (row stride C, rows overlapping).  Every layer is a GEMM on
// such views:
//   forward      Z   = im2col(Y_prev) . W^T + b      W  [Cout][5][Cin]
//   data grad    dY  = im2col(dZ) . Wf^T             Wf [Cin][5][Cout], Wf[ci][t][co] = W[co][4-t][ci]
//   weight grad  dW^T = im2col(Y_prev)^T . dZ         (K = positions)
// with the epilogues fused: bias + GELU (keeping Z for the backward pass),
// GELU' times the incoming gradient, and a row mask that keeps padding rows
// at zero (so the next layer's window reads zeros there, and no gradient
// flows from them).
//
// The GEMM is a 128x128x32 tile per CTA, 8 warps of 64x32, mma.sync
// m16n8k16 bf16 -> fp32 fed by ldmatrix (.trans for operands stored with M
// or N contiguous), three cp.async stages.  The database scoring GEMM is
// FP8 e4m3 (mma.sync m16n8k32): each CTA keeps 128 queries' embeddings in
// shared memory and streams 128-row database tiles, and its epilogue appends
// every (query, row) whose score reaches the query's threshold to that
// query's candidate list -- the [queries x database] score matrix is never
// written.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>

#include "common.cuh"

namespace sseqs {
namespace emb {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3, GEMM_THREADS = 256;
constexpr int LDK = BK + 8;        // [row][k] tile row, elements (80 B: ldmatrix conflict-free)
constexpr int LDR = BM + 8;        // [k][row] tile row, elements (272 B)

enum Epi : int {
  EPI_F32 = 0,          // C (fp32) = acc
  EPI_BF16 = 1,         // C (bf16) = acc  (masked rows -> 0)
  EPI_BIAS_GELU = 2,    // Z = acc + bias (bf16, C2), C = gelu(Z) (bf16); masked rows -> 0
  EPI_GELU_GRAD = 3,    // C (bf16) = acc * gelu'(aux);  masked rows -> 0
  EPI_F32_ADD = 4,      // C (fp32) += acc (atomic; split-K partial sums)
  EPI_BIAS_GELU_RES = 5,  // as 2, then C += res (bf16, C's stride): a residual connection
  EPI_GELU_GRAD_RES = 6,  // G = acc + res -> C2 (bf16), C = G * gelu'(aux); masked rows -> 0
};

// tanh by the hardware approximation (one MUFU instruction, relative error
// about 2^-11): GELU's outputs are rounded to bf16 (2^-8) right after.
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_f(float z) {
  const float u = 0.7978845608f * (z + 0.044715f * z * z * z);
  return 0.5f * z * (1.f + tanh_fast(u));
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float u = 0.7978845608f * (z + 0.044715f * z * z * z);
  const float t = tanh_fast(u);
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * 0.7978845608f * (1.f + 0.134145f * z * z);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool pred) {
  const int n = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

struct GemmArgs {
  int64_t M, N, K;
  const __nv_bfloat16* A;
  int64_t lda;
  const __nv_bfloat16* B;
  int64_t ldb;
  void* C;
  int64_t ldc;
  __nv_bfloat16* C2;          // EPI_BIAS_GELU: pre-activation
  const float* bias;
  const __nv_bfloat16* aux;   // EPI_GELU_GRAD(_RES): pre-activation
  const uint8_t* row_mask;    // nullable: 0 = padding row
  const __nv_bfloat16* res;   // EPI_*_RES: residual term
};

// A_T: A stored [K][M] (element (m,k) at A[k*lda + m]) instead of [M][K].
// B_T: B stored [K][N] instead of [N][K].
template <bool A_T, bool B_T, int EPI>
__global__ void __launch_bounds__(GEMM_THREADS) gemm_kernel(GemmArgs g) {
  constexpr int A_TILE = A_T ? BK * LDR : BM * LDK;
  constexpr int B_TILE = B_T ? BK * LDR : BN * LDK;
  extern __shared__ __align__(16) unsigned char gsm[];
  __nv_bfloat16* sA = reinterpret_cast<__nv_bfloat16*>(gsm);
  __nv_bfloat16* sB = sA + STAGES * A_TILE;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;          // 2 x 4 warps of 64 x 32
  const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
  // split-K: blockIdx.z takes k tiles [kt_lo, kt_hi)
  const int64_t kt_all = g.K / BK;
  const int64_t kt_per = (kt_all + gridDim.z - 1) / gridDim.z;
  const int64_t kt_lo = (int64_t)blockIdx.z * kt_per;
  const int64_t kt_hi = kt_lo + kt_per < kt_all ? kt_lo + kt_per : kt_all;
  const int64_t ktiles = kt_hi > kt_lo ? kt_hi - kt_lo : 0;

  auto load_tile = [&](int stage, int64_t kt) {
    const int64_t k0 = (kt_lo + kt) * BK;
    __nv_bfloat16* a = sA + stage * A_TILE;
    __nv_bfloat16* b = sB + stage * B_TILE;
#pragma unroll
    for (int it = 0; it < 2; ++it) {
      const int c = tid + it * GEMM_THREADS;        // 512 16-byte chunks per operand
      if (!A_T) {
        const int r = c >> 2, kc = (c & 3) * 8;
        const int64_t m = m0 + r;
        const bool ok = m < g.M;
        cp_async16(a + r * LDK + kc, g.A + (ok ? m : 0) * g.lda + k0 + kc, ok);
      } else {
        const int r = c >> 4, mc = (c & 15) * 8;
        const int64_t m = m0 + mc;
        const bool ok = m < g.M;
        cp_async16(a + r * LDR + mc, g.A + (k0 + r) * g.lda + (ok ? m : 0), ok);
      }
      if (!B_T) {
        const int r = c >> 2, kc = (c & 3) * 8;
        const int64_t n = n0 + r;
        const bool ok = n < g.N;
        cp_async16(b + r * LDK + kc, g.B + (ok ? n : 0) * g.ldb + k0 + kc, ok);
      } else {
        const int r = c >> 4, nc = (c & 15) * 8;
        const int64_t n = n0 + nc;
        const bool ok = n < g.N;
        cp_async16(b + r * LDR + nc, g.B + (k0 + r) * g.ldb + (ok ? n : 0), ok);
      }
    }
  };

  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) load_tile(s, s);
    cp_commit();
  }

  for (int64_t kt = 0; kt < ktiles; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    {
      const int64_t nk = kt + STAGES - 1;
      if (nk < ktiles) load_tile((int)(nk % STAGES), nk);
      cp_commit();
    }
    const __nv_bfloat16* a = sA + (kt % STAGES) * A_TILE;
    const __nv_bfloat16* b = sB + (kt % STAGES) * B_TILE;
#pragma unroll
    for (int ks = 0; ks < BK; ks += 16) {
      uint32_t af[4][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int mr = wm * 64 + i * 16;
        if (!A_T) {
          ldsm_x4(af[i], a + (mr + (lane & 15)) * LDK + ks + (lane >> 4) * 8);
        } else {
          const int j = lane >> 3, r = lane & 7;   // matrix j: m-half j&1, k-half j>>1
          ldsm_x4_t(af[i], a + (ks + (j >> 1) * 8 + r) * LDR + mr + (j & 1) * 8);
        }
      }
#pragma unroll
      for (int jp = 0; jp < 2; ++jp) {
        const int nr = wn * 32 + jp * 16;
        uint32_t t[4];
        const int j = lane >> 3, r = lane & 7;     // matrix j: n-half j>>1, k-half j&1
        if (!B_T) ldsm_x4(t, b + (nr + (j >> 1) * 8 + r) * LDK + ks + (j & 1) * 8);
        else ldsm_x4_t(t, b + (ks + (j & 1) * 8 + r) * LDR + nr + (j >> 1) * 8);
        bf[2 * jp][0] = t[0];
        bf[2 * jp][1] = t[1];
        bf[2 * jp + 1][0] = t[2];
        bf[2 * jp + 1][1] = t[3];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bf[j][0], bf[j][1]);
    }
  }
  cp_wait<0>();

  // epilogue
#pragma unroll
  for (int i = 0; i < 4; ++i) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t m = m0 + wm * 64 + i * 16 + (lane >> 2) + h * 8;
      if (m >= g.M) continue;
      const bool keep = g.row_mask ? g.row_mask[m] != 0 : true;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t n = n0 + wn * 32 + j * 8 + (lane & 3) * 2;
        if (n >= g.N) continue;
        const bool two = n + 1 < g.N;
        float v0 = acc[i][j][2 * h], v1 = acc[i][j][2 * h + 1];
        if (EPI == EPI_F32) {
          float* c = reinterpret_cast<float*>(g.C) + m * g.ldc + n;
          c[0] = v0;
          if (two) c[1] = v1;
        } else if (EPI == EPI_F32_ADD) {
          float* c = reinterpret_cast<float*>(g.C) + m * g.ldc + n;
          atomicAdd(c, v0);
          if (two) atomicAdd(c + 1, v1);
        } else if (EPI == EPI_BF16) {
          if (!keep) v0 = v1 = 0.f;
          __nv_bfloat16* c = reinterpret_cast<__nv_bfloat16*>(g.C) + m * g.ldc + n;
          c[0] = __float2bfloat16_rn(v0);
          if (two) c[1] = __float2bfloat16_rn(v1);
        } else if (EPI == EPI_BIAS_GELU || EPI == EPI_BIAS_GELU_RES) {
          const float z0 = v0 + g.bias[n], z1 = two ? v1 + g.bias[n + 1] : 0.f;
          __nv_bfloat16* c = reinterpret_cast<__nv_bfloat16*>(g.C) + m * g.ldc + n;
          __nv_bfloat16* z = g.C2 + m * g.ldc + n;
          const __nv_bfloat16 zb0 = __float2bfloat16_rn(keep ? z0 : 0.f);
          const __nv_bfloat16 zb1 = __float2bfloat16_rn(keep ? z1 : 0.f);
          float r0 = 0.f, r1 = 0.f;
          if (EPI == EPI_BIAS_GELU_RES) {
            const __nv_bfloat16* rs = g.res + m * g.ldc + n;
            r0 = __bfloat162float(rs[0]);
            r1 = two ? __bfloat162float(rs[1]) : 0.f;
          }
          if (g.C2) z[0] = zb0;
          c[0] = __float2bfloat16_rn(keep ? gelu_f(__bfloat162float(zb0)) + r0 : 0.f);
          if (two) {
            if (g.C2) z[1] = zb1;
            c[1] = __float2bfloat16_rn(keep ? gelu_f(__bfloat162float(zb1)) + r1 : 0.f);
          }
        } else if (EPI == EPI_GELU_GRAD_RES) {
          const __nv_bfloat16* ax = g.aux + m * g.ldc + n;
          const __nv_bfloat16* rs = g.res + m * g.ldc + n;
          __nv_bfloat16* c = reinterpret_cast<__nv_bfloat16*>(g.C) + m * g.ldc + n;
          __nv_bfloat16* gg = g.C2 + m * g.ldc + n;
          const __nv_bfloat16 g0 = __float2bfloat16_rn(keep ? v0 + __bfloat162float(rs[0]) : 0.f);
          gg[0] = g0;
          c[0] = __float2bfloat16_rn(keep ? __bfloat162float(g0) *
                                                gelu_grad(__bfloat162float(ax[0])) : 0.f);
          if (two) {
            const __nv_bfloat16 g1 =
                __float2bfloat16_rn(keep ? v1 + __bfloat162float(rs[1]) : 0.f);
            gg[1] = g1;
            c[1] = __float2bfloat16_rn(keep ? __bfloat162float(g1) *
                                                  gelu_grad(__bfloat162float(ax[1])) : 0.f);
          }
        } else {   // EPI_GELU_GRAD
          const __nv_bfloat16* ax = g.aux + m * g.ldc + n;
          __nv_bfloat16* c = reinterpret_cast<__nv_bfloat16*>(g.C) + m * g.ldc + n;
          c[0] = __float2bfloat16_rn(keep ? v0 * gelu_grad(__bfloat162float(ax[0])) : 0.f);
          if (two) c[1] = __float2bfloat16_rn(keep ? v1 * gelu_grad(__bfloat162float(ax[1])) : 0.f);
        }
      }
    }
  }
}

template <bool A_T, bool B_T, int EPI>
int launch_gemm(const GemmArgs& g, cudaStream_t stream, int splits = 1) {
  static_assert(EPI >= 0 && EPI <= 6, "epilogue");
  constexpr int A_TILE = A_T ? BK * LDR : BM * LDK;
  constexpr int B_TILE = B_T ? BK * LDR : BN * LDK;
  constexpr size_t smem = sizeof(__nv_bfloat16) * STAGES * (A_TILE + B_TILE);
  auto fn = gemm_kernel<A_T, B_T, EPI>;
  if (cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return SSEQS_ERR_CUDA;
  if (splits > 65535) return SSEQS_ERR_UNSUPPORTED;
  // blockIdx.y counts M tiles, at most 65535 per launch: longer M runs as
  // several launches over row ranges (the operands and outputs offset)
  constexpr int64_t kRows = (int64_t)65535 * BM;
  constexpr int64_t c_elem = (EPI == EPI_F32 || EPI == EPI_F32_ADD) ? 4 : 2;
  for (int64_t m0 = 0; m0 < g.M; m0 += kRows) {
    GemmArgs p = g;
    p.M = std::min(kRows, g.M - m0);
    p.A = A_T ? g.A + m0 : g.A + m0 * g.lda;
    p.C = static_cast<char*>(g.C) + m0 * g.ldc * c_elem;
    if (g.C2) p.C2 = g.C2 + m0 * g.ldc;
    if (g.aux) p.aux = g.aux + m0 * g.ldc;
    if (g.res) p.res = g.res + m0 * g.ldc;
    if (g.row_mask) p.row_mask = g.row_mask + m0;
    const dim3 grid((unsigned)((p.N + BN - 1) / BN), (unsigned)((p.M + BM - 1) / BM),
                    (unsigned)splits);
    { fn<<<grid, GEMM_THREADS, smem, stream>>>(p); count_launches(1); }
    const int st = status_of(cudaGetLastError());
    if (st != SSEQS_OK) return st;
  }
  return SSEQS_OK;
}

// ------------------------------------------------------- tcgen05 GEMM
// The N = 256 conv GEMMs (forward of layers 2-4, data gradients of layers
// 1-3) on the 5th-generation tensor cores: C[128 x 256] per CTA accumulates
// in tensor memory (256 fp32 columns x 128 lanes), fed from shared memory.
//
// Shared-memory operands use the K-major, no-swizzle canonical layout of
// the MMA: 8-row x 16-byte "core matrices" (8 rows x 8 bf16 of K), the
// core matrices of one 8-row group along K 128 bytes apart (leading byte
// offset) and consecutive 8-row groups 1024 bytes apart (stride byte
// offset) for a 64-wide K tile: element (row r, k) of a tile sits at
// (r/8)*1024 + (k/8)*128 + (r%8)*16 + (k%8)*2.  cp.async writes the tiles
// (two stages of A 16 KB + B 32 KB, two CTAs per SM, each with 256 of the
// SM's 512 tensor-memory columns); one thread issues the MMAs of a
// stage (K 16 each) and commits them to the stage's mbarrier, which the
// loaders wait on before reusing the stage.  Every wait is bounded: a
// wait that runs out sets *err, the kernel stops issuing work and waits
// (bounded) for the MMAs it already issued before it frees the tensor
// memory.  The
// epilogue reads the accumulators with tcgen05.ld (warp w reads lanes
// 32(w%4)..+31 = output rows, warps 0-3 columns 0-127 and warps 4-7
// columns 128-255) and applies the same fused epilogues as the mma.sync
// kernel.
constexpr int TC_BM = 128, TC_BN = 256, TC_BK = 64, TC_STAGES = 2, TC_THREADS = 256;
constexpr int TC_A_BYTES = TC_BM * TC_BK * 2, TC_B_BYTES = TC_BN * TC_BK * 2;
constexpr int TC_STAGE_BYTES = TC_A_BYTES + TC_B_BYTES;
constexpr size_t TC_SMEM = (size_t)TC_STAGES * TC_STAGE_BYTES + 1024;
constexpr unsigned kWaitLimit = 1u << 26;

// Shared-memory matrix descriptor: start, leading (K) and stride (MN)
// byte offsets in 16-byte units, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;            // version
  return d;                          // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor, kind::f16: fp32 accumulate, bf16 A and B, both
// K-major, M = 128, N = 256.
constexpr uint32_t kIdescBf16 = (1u << 4)            // D format F32
                              | (1u << 7)            // A format BF16
                              | (1u << 10)           // B format BF16
                              | ((uint32_t)(TC_BN >> 3) << 17)
                              | ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (unsigned i = 0; i < kWaitLimit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}

template <int EPI>
__global__ void __launch_bounds__(TC_THREADS, 2) gemm_tc_kernel(GemmArgs g, int* err) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  // align the tile area to 1024 bytes
  const uint32_t raw = smem_u32(tsm);
  unsigned char* tiles = tsm + ((1024 - (raw & 1023)) & 1023);
  __shared__ __align__(8) uint64_t mbar[TC_STAGES], drain;
  __shared__ uint32_t tmem_base_s;
  __shared__ int abort_s;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = (int64_t)blockIdx.x * TC_BM;
  const int64_t ktiles = g.K / TC_BK;

  if (warp == 0) {
    const uint32_t dst = smem_u32(&tmem_base_s);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(dst), "r"(TC_BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < TC_STAGES; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&mbar[s])), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&drain)), "r"(1));
    abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;

  auto load_stage = [&](int stage, int64_t kt) {
    unsigned char* a = tiles + stage * TC_STAGE_BYTES;
    unsigned char* b = a + TC_A_BYTES;
    const int64_t k0 = kt * TC_BK;
    // A: 128 rows x 8 chunks of 16 B
    for (int c = tid; c < TC_BM * 8; c += TC_THREADS) {
      const int r = c >> 3, kc = c & 7;
      const int64_t m = m0 + r;
      const bool ok = m < g.M;
      cp_async16(a + (r >> 3) * 1024 + kc * 128 + (r & 7) * 16,
                 g.A + (ok ? m : 0) * g.lda + k0 + kc * 8, ok);
    }
    // B: 256 rows x 8 chunks
    for (int c = tid; c < TC_BN * 8; c += TC_THREADS) {
      const int r = c >> 3, kc = c & 7;
      cp_async16(b + (r >> 3) * 1024 + kc * 128 + (r & 7) * 16,
                 g.B + (int64_t)r * g.ldb + k0 + kc * 8, true);
    }
  };

  // prologue: stages 0 .. S-2
  for (int s = 0; s < TC_STAGES - 1; ++s) {
    if (s < ktiles) load_stage(s, s);
    cp_commit();
  }
  uint32_t phase[TC_STAGES] = {};
  bool ok = true;
  for (int64_t kt = 0; kt < ktiles && ok; ++kt) {
    const int stage = (int)(kt % TC_STAGES);
    // refill the stage of tile kt + S - 1 once the MMAs that read it (tile
    // kt - 1) are done
    {
      const int64_t nk = kt + TC_STAGES - 1;
      const int ns = (int)(nk % TC_STAGES);
      if (nk < ktiles) {
        if (kt >= 1) {
          if (!mbar_wait(smem_u32(&mbar[ns]), phase[ns])) { if (tid == 0) abort_s = 1; }
          phase[ns] ^= 1;
        }
        load_stage(ns, nk);
      }
      cp_commit();
    }
    cp_wait<TC_STAGES - 1>();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (abort_s) { ok = false; break; }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(tiles + stage * TC_STAGE_BYTES);
      const uint32_t b0 = a0 + TC_A_BYTES;
#pragma unroll
      for (int ks = 0; ks < TC_BK / 16; ++ks) {
        const uint64_t da = umma_desc(a0 + ks * 256, 128, 1024);
        const uint64_t db = umma_desc(b0 + ks * 256, 128, 1024);
        const uint32_t acc = (kt > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
            :: "r"(tmem), "l"(da), "l"(db), "r"(kIdescBf16), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(smem_u32(&mbar[stage])) : "memory");
    }
  }
  cp_wait<0>();
  // wait for the last tile's MMAs (they complete in order, so this covers all)
  if (ok && ktiles > 0) {
    const int ls = (int)((ktiles - 1) % TC_STAGES);
    // the stage's barrier has completed one phase per tile it held; the
    // parity of the last one is the number of earlier completions mod 2
    const uint32_t par = (uint32_t)(((ktiles - 1) / TC_STAGES) & 1);
    if (!mbar_wait(smem_u32(&mbar[ls]), par)) ok = false;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!ok) {
    // MMAs already issued may still run: before the tensor memory and the
    // stages are given up, wait (bounded) until every one of them is done
    if (tid == 0) {
      atomicExch(err, 1);
      if (ktiles > 0) {
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(smem_u32(&drain)) : "memory");
        mbar_wait(smem_u32(&drain), 0);
      }
    }
  } else {
    const int wq = warp & 3;                       // lanes 32*wq .. +31
    const int64_t m = m0 + wq * 32 + lane;
    const bool row_ok = m < g.M;
    const bool keep = row_ok && (g.row_mask ? g.row_mask[m] != 0 : true);
    const int cbeg = (warp >> 2) * (TC_BN / 2);
#pragma unroll 1
    for (int c0 = cbeg; c0 < cbeg + TC_BN / 2; c0 += 32) {
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
          "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
            "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
            "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
            "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (!row_ok) continue;
      // this row's 32 residual / pre-activation values, 16 bytes at a time
      __align__(16) __nv_bfloat16 rs[32], ax[32];
      if (EPI == EPI_BIAS_GELU_RES || EPI == EPI_GELU_GRAD_RES) {
        const uint4* src = reinterpret_cast<const uint4*>(g.res + m * g.ldc + c0);
#pragma unroll
        for (int q = 0; q < 4; ++q) reinterpret_cast<uint4*>(rs)[q] = src[q];
      }
      if (EPI == EPI_GELU_GRAD || EPI == EPI_GELU_GRAD_RES) {
        const uint4* src = reinterpret_cast<const uint4*>(g.aux + m * g.ldc + c0);
#pragma unroll
        for (int q = 0; q < 4; ++q) reinterpret_cast<uint4*>(ax)[q] = src[q];
      }
      __align__(16) __nv_bfloat16 outc[32], outz[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int64_t n = c0 + j;
        const float acc = __uint_as_float(v[j]);
        float cval = 0.f, zval = 0.f;
        if (EPI == EPI_BF16) {
          cval = keep ? acc : 0.f;
        } else if (EPI == EPI_BIAS_GELU || EPI == EPI_BIAS_GELU_RES) {
          const __nv_bfloat16 zb = __float2bfloat16_rn(keep ? acc + g.bias[n] : 0.f);
          zval = __bfloat162float(zb);
          const float r = (EPI == EPI_BIAS_GELU_RES) ? __bfloat162float(rs[j]) : 0.f;
          cval = keep ? gelu_f(zval) + r : 0.f;
        } else if (EPI == EPI_GELU_GRAD) {
          cval = keep ? acc * gelu_grad(__bfloat162float(ax[j])) : 0.f;
        } else {   // EPI_GELU_GRAD_RES
          const __nv_bfloat16 gb = __float2bfloat16_rn(keep ? acc + __bfloat162float(rs[j]) : 0.f);
          zval = __bfloat162float(gb);
          cval = keep ? zval * gelu_grad(__bfloat162float(ax[j])) : 0.f;
        }
        outc[j] = __float2bfloat16_rn(cval);
        outz[j] = __float2bfloat16_rn(zval);
      }
      uint4* dc = reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(g.C) + m * g.ldc + c0);
      const uint4* sc = reinterpret_cast<const uint4*>(outc);
#pragma unroll
      for (int q = 0; q < 4; ++q) dc[q] = sc[q];
      if ((EPI == EPI_BIAS_GELU || EPI == EPI_BIAS_GELU_RES || EPI == EPI_GELU_GRAD_RES) && g.C2) {
        uint4* dz = reinterpret_cast<uint4*>(g.C2 + m * g.ldc + c0);
        const uint4* sz = reinterpret_cast<const uint4*>(outz);
#pragma unroll
        for (int q = 0; q < 4; ++q) dz[q] = sz[q];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TC_BN));
}

// ------------------------------------------- tcgen05 GEMM, TMA-fed, persistent
// The same N = 256 GEMMs, warp-specialised: warp 0 (one thread) loads the
// tiles with TMA (cp.async.bulk.tensor, 128-byte swizzle, no multicast:
// operands are this GPU's own memory), warp 1 (one thread) issues the MMAs,
// warps 2-9 drain the accumulators.  Four stages of A (128 x 64 bf16) and B
// (256 x 64) -- 192 KB -- and two 128 x 256 fp32 accumulators in tensor
// memory (all 512 columns), so the epilogue of one M tile runs while the
// next accumulates.  CTAs are persistent (one per SM) and take M tiles in
// turn.  Barriers: full[s] (TMA bytes landed), empty[s] (the MMAs that read
// stage s are done), acc_full[b] (accumulator b complete), acc_empty[b]
// (its 8 epilogue warps have read it).  Every wait is bounded; one that runs
// out sets *err, raises the CTA's abort flag and the roles stop issuing work;
// before the tensor memory is freed the MMA thread waits (bounded) for its
// last MMAs and the loader for its outstanding loads.
//
// A may be an overlapping row view (the conv GEMMs: row m of im2col(Y) starts
// lda elements after row m-1 and spans K = 5 * lda): its tensor map is the
// 2D array of lda-wide rows, and the K tile at k0 is the box at column
// k0 % lda of row m0 + k0 / lda (a tile never crosses a row when lda % 64 ==
// 0; for lda >= K it is the plain matrix).
constexpr int WS_STAGES = 4, WS_EPI_WARPS = 8, WS_THREADS = 32 * (2 + WS_EPI_WARPS);
constexpr size_t WS_SMEM = (size_t)WS_STAGES * TC_STAGE_BYTES + 1024;

// Shared-memory matrix descriptor, K-major with the 128-byte swizzle: rows of
// 128 bytes (64 bf16 of K), 8-row swizzle atoms 1024 bytes apart.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                  // leading byte offset (unused for this layout)
  d |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                  // version
  d |= (uint64_t)2 << 61;                  // layout: 128-byte swizzle
  return d;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];"
      :: "r"(dst), "l"(map), "r"(x), "r"(y), "r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mbar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(mbar) : "memory");
}

// Fused epilogue of one row's 32 accumulator columns c0 .. c0 + 31.
template <int EPI>
__device__ __forceinline__ void epi_store32(const GemmArgs& g, int64_t m, bool keep, int c0,
                                            const uint32_t (&v)[32]) {
  __align__(16) __nv_bfloat16 rs[32], ax[32];
  if (EPI == EPI_BIAS_GELU_RES || EPI == EPI_GELU_GRAD_RES) {
    const uint4* src = reinterpret_cast<const uint4*>(g.res + m * g.ldc + c0);
#pragma unroll
    for (int q = 0; q < 4; ++q) reinterpret_cast<uint4*>(rs)[q] = src[q];
  }
  if (EPI == EPI_GELU_GRAD || EPI == EPI_GELU_GRAD_RES) {
    const uint4* src = reinterpret_cast<const uint4*>(g.aux + m * g.ldc + c0);
#pragma unroll
    for (int q = 0; q < 4; ++q) reinterpret_cast<uint4*>(ax)[q] = src[q];
  }
  __align__(16) __nv_bfloat16 outc[32], outz[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const int64_t n = c0 + j;
    const float acc = __uint_as_float(v[j]);
    float cval = 0.f, zval = 0.f;
    if (EPI == EPI_BF16) {
      cval = keep ? acc : 0.f;
    } else if (EPI == EPI_BIAS_GELU || EPI == EPI_BIAS_GELU_RES) {
      const __nv_bfloat16 zb = __float2bfloat16_rn(keep ? acc + g.bias[n] : 0.f);
      zval = __bfloat162float(zb);
      const float r = (EPI == EPI_BIAS_GELU_RES) ? __bfloat162float(rs[j]) : 0.f;
      cval = keep ? gelu_f(zval) + r : 0.f;
    } else if (EPI == EPI_GELU_GRAD) {
      cval = keep ? acc * gelu_grad(__bfloat162float(ax[j])) : 0.f;
    } else {   // EPI_GELU_GRAD_RES
      const __nv_bfloat16 gb = __float2bfloat16_rn(keep ? acc + __bfloat162float(rs[j]) : 0.f);
      zval = __bfloat162float(gb);
      cval = keep ? zval * gelu_grad(__bfloat162float(ax[j])) : 0.f;
    }
    outc[j] = __float2bfloat16_rn(cval);
    outz[j] = __float2bfloat16_rn(zval);
  }
  uint4* dc = reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(g.C) + m * g.ldc + c0);
  const uint4* sc = reinterpret_cast<const uint4*>(outc);
#pragma unroll
  for (int q = 0; q < 4; ++q) dc[q] = sc[q];
  // the pre-activation (C2) is optional for the forward epilogues: only the
  // backward pass reads it
  if ((EPI == EPI_BIAS_GELU || EPI == EPI_BIAS_GELU_RES || EPI == EPI_GELU_GRAD_RES) && g.C2) {
    uint4* dz = reinterpret_cast<uint4*>(g.C2 + m * g.ldc + c0);
    const uint4* sz = reinterpret_cast<const uint4*>(outz);
#pragma unroll
    for (int q = 0; q < 4; ++q) dz[q] = sz[q];
  }
}

template <int EPI>
__global__ void __launch_bounds__(WS_THREADS, 1)
    gemm_ws_kernel(const __grid_constant__ CUtensorMap map_a,
                   const __grid_constant__ CUtensorMap map_b, GemmArgs g, int a_row_len,
                   int* err) {
  extern __shared__ __align__(1024) unsigned char wsm[];
  const uint32_t raw = smem_u32(wsm);
  unsigned char* tiles = wsm + ((1024 - (raw & 1023)) & 1023);
  __shared__ __align__(8) uint64_t full[WS_STAGES], empty[WS_STAGES];
  __shared__ __align__(8) uint64_t acc_full[2], acc_empty[2], mma_done;
  __shared__ uint32_t tmem_base_s;
  __shared__ volatile int abort_s;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t ntiles = (g.M + TC_BM - 1) / TC_BM;
  const int ktiles = (int)(g.K / TC_BK);

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&tmem_base_s)), "r"(2 * TC_BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < WS_STAGES; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&full[s])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&empty[s])), "r"(1));
    }
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&acc_full[b])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                   :: "r"(smem_u32(&acc_empty[b])), "r"(WS_EPI_WARPS));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&mma_done)), "r"(1));
    abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  auto fail = [&]() {
    abort_s = 1;
    atomicExch(err, 1);
  };

  if (warp == 0) {
    // ------------------------------------------------------------ loader
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" :: "l"(&map_a) : "memory");
      asm volatile("prefetch.tensormap [%0];" :: "l"(&map_b) : "memory");
      int stage = 0;
      uint32_t phase = 0;
      uint32_t loads[WS_STAGES] = {};      // loads issued into each stage
      for (int64_t t = blockIdx.x; t < ntiles && !abort_s; t += gridDim.x) {
        const int m0 = (int)(t * TC_BM);
        for (int kt = 0; kt < ktiles && !abort_s; ++kt) {
          if (!mbar_wait(smem_u32(&empty[stage]), phase ^ 1)) { fail(); break; }
          const uint32_t fb = smem_u32(&full[stage]);
          mbar_expect_tx(fb, (uint32_t)TC_STAGE_BYTES);
          const uint32_t a = smem_u32(tiles + stage * TC_STAGE_BYTES);
          const int k0 = kt * TC_BK;
          tma_load_2d(a, &map_a, k0 % a_row_len, m0 + k0 / a_row_len, fb);
          tma_load_2d(a + TC_A_BYTES, &map_b, k0, 0, fb);
          ++loads[stage];
          if (++stage == WS_STAGES) { stage = 0; phase ^= 1; }
        }
      }
      // before exit every issued load has landed: on the normal path the
      // MMAs consumed them all; after an abort, wait (bounded) for the last
      // load of each stage, which completes phase loads - 1 of its barrier
      if (abort_s) {
        for (int s2 = 0; s2 < WS_STAGES; ++s2)
          if (loads[s2] > 0) mbar_wait(smem_u32(&full[s2]), (loads[s2] - 1) & 1u);
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issue
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int b = 0;
      uint32_t acc_phase = 0;
      bool any = false;
      for (int64_t t = blockIdx.x; t < ntiles && !abort_s; t += gridDim.x) {
        if (!mbar_wait(smem_u32(&acc_empty[b]), acc_phase ^ 1)) { fail(); break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(b * TC_BN);
        for (int kt = 0; kt < ktiles; ++kt) {
          if (!mbar_wait(smem_u32(&full[stage]), phase)) { fail(); break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(tiles + stage * TC_STAGE_BYTES);
          const uint32_t b0 = a0 + TC_A_BYTES;
#pragma unroll
          for (int ks = 0; ks < TC_BK / 16; ++ks) {
            const uint64_t da = umma_desc_sw128(a0 + ks * 32);
            const uint64_t db = umma_desc_sw128(b0 + ks * 32);
            const uint32_t accum = (kt > 0 || ks > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                :: "r"(acc), "l"(da), "l"(db), "r"(kIdescBf16), "r"(accum));
          }
          any = true;
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                       :: "r"(smem_u32(&empty[stage])) : "memory");
          if (++stage == WS_STAGES) { stage = 0; phase ^= 1; }
        }
        if (abort_s) break;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(smem_u32(&acc_full[b])) : "memory");
        if (++b == 2) { b = 0; acc_phase ^= 1; }
      }
      // every MMA issued is complete before the tensor memory is freed
      if (any) {
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(smem_u32(&mma_done)) : "memory");
        if (!mbar_wait(smem_u32(&mma_done), 0)) fail();
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int e = warp - 2;
    const int q = warp & 3;                      // tensor-memory lanes 32q .. 32q + 31
    const int cbeg = (e >> 2) * (TC_BN / 2);     // columns [cbeg, cbeg + 128)
    int b = 0;
    uint32_t acc_phase = 0;
    for (int64_t t = blockIdx.x; t < ntiles && !abort_s; t += gridDim.x) {
      if (!mbar_wait(smem_u32(&acc_full[b]), acc_phase)) { if (lane == 0) fail(); break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int64_t m = t * TC_BM + q * 32 + lane;
      const bool row_ok = m < g.M;
      const bool keep = row_ok && (g.row_mask ? g.row_mask[m] != 0 : true);
#pragma unroll 1
      for (int c0 = cbeg; c0 < cbeg + TC_BN / 2; c0 += 32) {
        uint32_t v[32];
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * TC_BN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
            "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
              "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
              "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
              "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
              "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
              "=r"(v[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row_ok) epi_store32<EPI>(g, m, keep, c0, v);
      }
      // this warp has read accumulator b: hand it back to the MMA thread
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acc_empty[b]));
      if (++b == 2) { b = 0; acc_phase ^= 1; }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(2 * TC_BN));
}

// ------------------------------------------------------------ elementwise
// First convolution as a table.  Its input rows are class embeddings, so
// the pre-activation of row p is b + sum_t T[t][cls[p-2+t]] with
// T[t][k] = E[k] . W1[:, t, :]^T (rows outside the layout and padding rows
// contribute nothing): a gather-add of five 256-wide rows instead of a K = 160
// GEMM.  Same epilogue as EPI_BIAS_GELU: Z = bf16(z), Y = GELU(Z); masked
// rows 0; Z optional.  A thread writes 8 channels of one row; T in shared
// memory (5 x 21 x D fp32).
__global__ void conv1_table_kernel(const uint8_t* cls, int64_t P, const float* T,
                                   const float* bias, const uint8_t* mask, int D,
                                   __nv_bfloat16* Y, __nv_bfloat16* Z) {
  extern __shared__ float4 t_sm[];
  float* Ts = reinterpret_cast<float*>(t_sm);
  for (int i = threadIdx.x; i < 5 * 21 * D / 4; i += blockDim.x)
    t_sm[i] = reinterpret_cast<const float4*>(T)[i];
  __syncthreads();
  const int per_row = D / 8;
  const int64_t total = P * per_row;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / per_row;
    const int c0 = (int)(i - p * per_row) * 8;
    const bool keep = mask ? mask[p] != 0 : true;
    float z[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) z[j] = bias[c0 + j];
#pragma unroll
    for (int t = 0; t < 5; ++t) {
      const int64_t q = p - 2 + t;
      const int k = (q >= 0 && q < P) ? cls[q] : 255;
      if (k < 21) {
        const float4* tr = reinterpret_cast<const float4*>(Ts + ((size_t)t * 21 + k) * D + c0);
        const float4 a = tr[0], b = tr[1];
        z[0] += a.x; z[1] += a.y; z[2] += a.z; z[3] += a.w;
        z[4] += b.x; z[5] += b.y; z[6] += b.z; z[7] += b.w;
      }
    }
    __align__(16) __nv_bfloat16 zy[8], yy[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      zy[j] = __float2bfloat16_rn(keep ? z[j] : 0.f);
      yy[j] = __float2bfloat16_rn(keep ? gelu_f(__bfloat162float(zy[j])) : 0.f);
    }
    *reinterpret_cast<uint4*>(Y + p * D + c0) = *reinterpret_cast<const uint4*>(yy);
    if (Z) *reinterpret_cast<uint4*>(Z + p * D + c0) = *reinterpret_cast<const uint4*>(zy);
  }
}

// X0[p][c] = E[cls[p]][c] for real rows (cls < 21), 0 for padding (cls 255).
__global__ void embed_lookup_kernel(const uint8_t* cls, int64_t P, const __nv_bfloat16* E, int D,
                                    __nv_bfloat16* X) {
  const int64_t total = P * D;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / D;
    const int c = (int)(i - p * D), k = cls[p];
    X[i] = k < 21 ? E[k * D + c] : __float2bfloat16_rn(0.f);
  }
}

// dE[cls[p]][c] += dX[p][c]
__global__ void embed_grad_kernel(const uint8_t* cls, int64_t P, const __nv_bfloat16* dX, int D,
                                  float* dE) {
  const int64_t total = P * D;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / D;
    const int c = (int)(i - p * D), k = cls[p];
    if (k < 21) atomicAdd(dE + k * D + c, __bfloat162float(dX[i]));
  }
}

// One block of D = blockDim.x threads per sequence: pooled = mean of its
// rows, emb = pooled / |pooled|.
__global__ void pool_normalize_kernel(const __nv_bfloat16* Y, const int64_t* start,
                                      const int32_t* len, float* pooled, float* emb,
                                      float* inv_norm) {
  const int s = blockIdx.x, c = threadIdx.x, D = blockDim.x;
  const int n = len[s];
  const __nv_bfloat16* y = Y + start[s] * D + c;
  float acc = 0.f;
  for (int p = 0; p < n; ++p) acc += __bfloat162float(y[(int64_t)p * D]);
  const float mean = n > 0 ? acc / (float)n : 0.f;
  __shared__ float red[32];
  float sq = mean * mean;
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
  if ((c & 31) == 0) red[c >> 5] = sq;
  __syncthreads();
  if (c < 32) {
    float v = c < (D >> 5) ? red[c] : 0.f;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (c == 0) red[0] = v;
  }
  __syncthreads();
  const float inv = rsqrtf(fmaxf(red[0], 1e-24f));
  pooled[(int64_t)s * D + c] = mean;
  emb[(int64_t)s * D + c] = mean * inv;
  if (c == 0) inv_norm[s] = inv;
}

// One warp per pair: pred = <e_a, e_b>; with weight w (1/B when no
// weights are given) loss += w (pred - y)^2, dE_a += 2 w (pred - y) e_b,
// dE_b likewise.
__global__ void pair_loss_kernel(const float* emb, int D, const int32_t* ia, const int32_t* ib,
                                 const float* y, const float* wt, int64_t B, float* dE,
                                 float* loss, float* pred_out) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= B) return;
  const float* ea = emb + (int64_t)ia[w] * D;
  const float* eb = emb + (int64_t)ib[w] * D;
  float d = 0.f;
  for (int c = lane; c < D; c += 32) d += ea[c] * eb[c];
  for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
  const float r = d - y[w];
  const float wgt = wt ? wt[w] : 1.f / (float)B;
  const float g = 2.f * r * wgt;
  if (lane == 0) {
    atomicAdd(loss, r * r * wgt);
    if (pred_out) pred_out[w] = d;
  }
  if (dE) {
    float* ga = dE + (int64_t)ia[w] * D;
    float* gb = dE + (int64_t)ib[w] * D;
    for (int c = lane; c < D; c += 32) {
      atomicAdd(ga + c, g * eb[c]);
      atomicAdd(gb + c, g * ea[c]);
    }
  }
}

// Gradient of the pooled, normalised embedding back to the last layer's
// pre-activation: dpooled = (dE - e <e, dE>) * inv_norm; each real row of
// sequence s gets dY = dpooled / len (stored in G when given), and
// dZ = dY * gelu'(Z).
__global__ void pool_backward_kernel(const float* emb, const float* dE, const float* inv_norm,
                                     const int64_t* start, const int32_t* len,
                                     const __nv_bfloat16* Z, __nv_bfloat16* dZ,
                                     __nv_bfloat16* G) {
  const int s = blockIdx.x, c = threadIdx.x, D = blockDim.x;
  const float e = emb[(int64_t)s * D + c], g = dE[(int64_t)s * D + c];
  __shared__ float red[32];
  float v = e * g;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((c & 31) == 0) red[c >> 5] = v;
  __syncthreads();
  if (c < 32) {
    float t = c < (D >> 5) ? red[c] : 0.f;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (c == 0) red[0] = t;
  }
  __syncthreads();
  const int n = len[s];
  const float dp = (g - e * red[0]) * inv_norm[s] / (float)max(n, 1);
  const int64_t base = start[s] * D + c;
  const __nv_bfloat16 gb = __float2bfloat16_rn(dp);
  for (int p = 0; p < n; ++p) {
    const int64_t i = base + (int64_t)p * D;
    dZ[i] = __float2bfloat16_rn(dp * gelu_grad(__bfloat162float(Z[i])));
    if (G) G[i] = gb;
  }
}

// db[c] += sum over rows of dZ[p][c] (block: 256 columns x a row range)
__global__ void bias_grad_kernel(const __nv_bfloat16* dZ, int64_t P, int D, float* db) {
  const int c = threadIdx.x + blockIdx.y * blockDim.x;
  if (c >= D) return;
  const int64_t rows = (P + gridDim.x - 1) / gridDim.x;
  const int64_t p0 = (int64_t)blockIdx.x * rows, p1 = min(P, p0 + rows);
  float acc = 0.f;
  for (int64_t p = p0; p < p1; ++p) acc += __bfloat162float(dZ[p * D + c]);
  atomicAdd(db + c, acc);
}

struct AdamArgs {
  float lr, b1, b2, eps, c1, c2;   // c1 = 1 - b1^t, c2 = 1 - b2^t
};
__device__ __forceinline__ float adam_step(float& w, float& m, float& v, float g,
                                           const AdamArgs& o) {
  m = o.b1 * m + (1.f - o.b1) * g;
  v = o.b2 * v + (1.f - o.b2) * g * g;
  w -= o.lr * (m / o.c1) / (sqrtf(v / o.c2) + o.eps);
  return w;
}

// Conv weight W[co][t][ci] (fp32 master + moments) from its gradient in the
// weight-grad GEMM's layout dWT[(t*Cin + ci)][co]; writes the bf16 copies
// W[co][t][ci] and Wf[ci][4-t][co].
__global__ void adam_conv_kernel(float* w, float* m, float* v, const float* dWT, int Cout,
                                 int Cin, AdamArgs o, __nv_bfloat16* Wb, __nv_bfloat16* Wf) {
  const int64_t total = (int64_t)Cout * 5 * Cin;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int co = (int)(i / (5 * Cin));
    const int r = (int)(i - (int64_t)co * 5 * Cin);
    const int t = r / Cin, ci = r - t * Cin;
    const float g = dWT[(int64_t)(t * Cin + ci) * Cout + co];
    const float nw = adam_step(w[i], m[i], v[i], g, o);
    const __nv_bfloat16 b = __float2bfloat16_rn(nw);
    Wb[i] = b;
    Wf[((int64_t)ci * 5 + (4 - t)) * Cout + co] = b;
  }
}

// Flat parameters (bias, residue embedding); optional bf16 copy.
__global__ void adam_flat_kernel(float* w, float* m, float* v, const float* g, int64_t n,
                                 AdamArgs o, __nv_bfloat16* wb) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float nw = adam_step(w[i], m[i], v[i], g[i], o);
    if (wb) wb[i] = __float2bfloat16_rn(nw);
  }
}

// e4m3 codes of scale * x
__global__ void quantize_e4m3_kernel(const float* x, int64_t n, float scale, uint8_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (uint8_t)__nv_cvt_float_to_fp8(scale * x[i], __NV_SATFINITE, __NV_E4M3);
}

// ------------------------------------------------------ FP8 score + select
constexpr int SK = 256;            // embedding width (bytes per e4m3 row)
constexpr int SLD = SK + 16;       // smem row stride (272 B: ldmatrix conflict-free)

__device__ __forceinline__ void mma_e4m3(float (&c)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.f32.e4m3.e4m3.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

struct SelArgs {
  const uint8_t* Q;        // [nq][256] e4m3
  int nq;
  const uint8_t* DB;       // [n][256] e4m3
  int64_t n;
  const float* tau;        // [nq] threshold on the raw dot product of the codes
  int32_t* count;          // [nq]
  int64_t* cand;           // [nq][cap] database rows
  float* cand_score;       // [nq][cap]
  int cap;
};

// CTA: 128 queries (blockIdx.y) x database tiles of 128 rows (blockIdx.x,
// gridDim.x apart).  Two database stages in flight.
__global__ void __launch_bounds__(GEMM_THREADS) score_select_kernel(SelArgs a) {
  extern __shared__ __align__(16) unsigned char ssm[];
  uint8_t* sQ = ssm;                         // [128][SLD]
  uint8_t* sD = ssm + 128 * SLD;             // [2][128][SLD]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;
  const int q0 = blockIdx.y * 128;
  // query tile (rows past nq are zero)
  for (int c = tid; c < 128 * (SK / 16); c += GEMM_THREADS) {
    const int r = c / (SK / 16), kc = (c % (SK / 16)) * 16;
    const bool ok = q0 + r < a.nq;
    cp_async16(sQ + r * SLD + kc, a.Q + (int64_t)(ok ? q0 + r : 0) * SK + kc, ok);
  }
  cp_commit();
  const int64_t ntiles = (a.n + 127) / 128;
  auto load_db = [&](int stage, int64_t tile) {
    uint8_t* d = sD + stage * 128 * SLD;
    for (int c = tid; c < 128 * (SK / 16); c += GEMM_THREADS) {
      const int r = c / (SK / 16), kc = (c % (SK / 16)) * 16;
      const int64_t row = tile * 128 + r;
      const bool ok = row < a.n;
      cp_async16(d + r * SLD + kc, a.DB + (ok ? row : 0) * SK + kc, ok);
    }
  };
  int64_t tile = blockIdx.x;
  if (tile < ntiles) load_db(0, tile);
  cp_commit();
  float tau[4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int q = q0 + wm * 64 + i * 16 + (lane >> 2) + h * 8;
      tau[i][h] = q < a.nq ? a.tau[q] : INFINITY;
    }
  int stage = 0;
  for (; tile < ntiles; tile += gridDim.x) {
    const int64_t next = tile + gridDim.x;
    if (next < ntiles) load_db(stage ^ 1, next);
    cp_commit();
    cp_wait<1>();
    __syncthreads();
    const uint8_t* d = sD + stage * 128 * SLD;
    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
#pragma unroll
    for (int ks = 0; ks < SK; ks += 32) {
      uint32_t af[4][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 4; ++i)
        ldsm_x4(af[i], sQ + (wm * 64 + i * 16 + (lane & 15)) * SLD + ks + (lane >> 4) * 16);
#pragma unroll
      for (int jp = 0; jp < 2; ++jp) {
        uint32_t t[4];
        const int j = lane >> 3, r = lane & 7;
        ldsm_x4(t, d + (wn * 32 + jp * 16 + (j >> 1) * 8 + r) * SLD + ks + (j & 1) * 16);
        bf[2 * jp][0] = t[0];
        bf[2 * jp][1] = t[1];
        bf[2 * jp + 1][0] = t[2];
        bf[2 * jp + 1][1] = t[3];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_e4m3(acc[i][j], af[i], bf[j][0], bf[j][1]);
    }
    // epilogue: append every score that reaches its query's threshold
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int q = q0 + wm * 64 + i * 16 + (lane >> 2) + h * 8;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const float v = acc[i][j][2 * h + e];
            const int64_t row = tile * 128 + wn * 32 + j * 8 + (lane & 3) * 2 + e;
            if (v >= tau[i][h] && row < a.n) {
              const int slot = atomicAdd(a.count + q, 1);
              if (slot < a.cap) {
                a.cand[(int64_t)q * a.cap + slot] = row;
                a.cand_score[(int64_t)q * a.cap + slot] = v;
              }
            }
          }
      }
    __syncthreads();     // stage is reloaded two tiles later
    stage ^= 1;
  }
  cp_wait<0>();
}

// Dense scores [nq][n] of the codes (for threshold sampling): one CTA per
// 128 queries x 128 rows.
__global__ void __launch_bounds__(GEMM_THREADS) score_dense_kernel(SelArgs a, float* out) {
  extern __shared__ __align__(16) unsigned char ssm[];
  uint8_t* sQ = ssm;
  uint8_t* sD = ssm + 128 * SLD;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;
  const int q0 = blockIdx.y * 128;
  const int64_t r0 = (int64_t)blockIdx.x * 128;
  for (int c = tid; c < 128 * (SK / 16); c += GEMM_THREADS) {
    const int r = c / (SK / 16), kc = (c % (SK / 16)) * 16;
    const bool okq = q0 + r < a.nq;
    cp_async16(sQ + r * SLD + kc, a.Q + (int64_t)(okq ? q0 + r : 0) * SK + kc, okq);
    const bool okd = r0 + r < a.n;
    cp_async16(sD + r * SLD + kc, a.DB + (okd ? r0 + r : 0) * SK + kc, okd);
  }
  cp_commit();
  cp_wait<0>();
  __syncthreads();
  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
#pragma unroll
  for (int ks = 0; ks < SK; ks += 32) {
    uint32_t af[4][4], bf[4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
      ldsm_x4(af[i], sQ + (wm * 64 + i * 16 + (lane & 15)) * SLD + ks + (lane >> 4) * 16);
#pragma unroll
    for (int jp = 0; jp < 2; ++jp) {
      uint32_t t[4];
      const int j = lane >> 3, r = lane & 7;
      ldsm_x4(t, sD + (wn * 32 + jp * 16 + (j >> 1) * 8 + r) * SLD + ks + (j & 1) * 16);
      bf[2 * jp][0] = t[0];
      bf[2 * jp][1] = t[1];
      bf[2 * jp + 1][0] = t[2];
      bf[2 * jp + 1][1] = t[3];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) mma_e4m3(acc[i][j], af[i], bf[j][0], bf[j][1]);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int q = q0 + wm * 64 + i * 16 + (lane >> 2) + h * 8;
      if (q >= a.nq) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int64_t row = r0 + wn * 32 + j * 8 + (lane & 3) * 2 + e;
          if (row < a.n) out[(int64_t)q * a.n + row] = acc[i][j][2 * h + e];
        }
    }
}

// ------------------------------------- FP8 score + select on tcgen05 (TMA)
// The same selection as score_select_kernel with the database rows as the
// M = 128 operand of tcgen05.mma kind::f8f6f4 and the query tile as N (the
// batch rounded up to 16, at most 256, so a small batch does not pay for a
// 128-query tile).  Persistent CTAs (one per SM) take 128-row database tiles
// in turn; warp 0 loads them with TMA (two 128 x 128-byte boxes per tile,
// 128-byte swizzle, no multicast: the codes are this GPU's own memory) into
// SEL_STAGES_MAX stages at most, warp 1 issues the eight K = 32 MMAs of a
// tile into one of two tensor-memory accumulators, and warps 2-9 read the
// other accumulator (warp w: rows 32(w%4)..+31, alternate 16-column groups)
// and append every (query, row) whose score reaches the query's threshold.
// The query tile is loaded once per CTA.  Waits are bounded as in
// gemm_ws_kernel and set the same error flag.
constexpr int SEL_STAGES_MAX = 6, SEL_EPI_WARPS = 8, SEL_THREADS = 32 * (2 + SEL_EPI_WARPS);
constexpr int SEL_TILE_BYTES = 128 * SK;          // 32 KB: two 16 KB K halves

__device__ __forceinline__ uint32_t sel_idesc(int N) {
  return (1u << 4)                                // D format F32; A, B format E4M3 (0)
       | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__global__ void __launch_bounds__(SEL_THREADS, 1)
    score_select_tc_kernel(const __grid_constant__ CUtensorMap map_db,
                           const __grid_constant__ CUtensorMap map_q, SelArgs a, int N,
                           int stages, int* err) {
  extern __shared__ __align__(1024) unsigned char xsm[];
  const uint32_t raw = smem_u32(xsm);
  unsigned char* base = xsm + ((1024 - (raw & 1023)) & 1023);
  unsigned char* sq = base;                                   // [2][N][128]
  unsigned char* tiles = base + (size_t)N * SK;               // [stages][2][128][128]
  __shared__ __align__(8) uint64_t full[SEL_STAGES_MAX], empty[SEL_STAGES_MAX];
  __shared__ __align__(8) uint64_t acc_full[2], acc_empty[2], q_full, mma_done;
  __shared__ float tau_s[256];
  __shared__ uint32_t tmem_base_s;
  __shared__ volatile int abort_s;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q0 = blockIdx.y * N;
  const int64_t ntiles = (a.n + 127) / 128;
  uint32_t tcols = 32;
  while (tcols < (uint32_t)(2 * N)) tcols <<= 1;

  for (int i = tid; i < N; i += blockDim.x)
    tau_s[i] = q0 + i < a.nq ? a.tau[q0 + i] : INFINITY;
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&tmem_base_s)), "r"(tcols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < stages; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&full[s])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&empty[s])), "r"(1));
    }
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&acc_full[b])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                   :: "r"(smem_u32(&acc_empty[b])), "r"(SEL_EPI_WARPS));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&q_full)), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&mma_done)), "r"(1));
    abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  auto fail = [&]() {
    abort_s = 1;
    atomicExch(err, 1);
  };

  if (warp == 0) {
    // ------------------------------------------------------------ loader
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" :: "l"(&map_db) : "memory");
      asm volatile("prefetch.tensormap [%0];" :: "l"(&map_q) : "memory");
      const uint32_t qb = smem_u32(&q_full);
      mbar_expect_tx(qb, (uint32_t)(N * SK));
      tma_load_2d(smem_u32(sq), &map_q, 0, q0, qb);
      tma_load_2d(smem_u32(sq + N * 128), &map_q, 128, q0, qb);
      int stage = 0;
      uint32_t phase = 0;
      uint32_t loads[SEL_STAGES_MAX] = {};
      for (int64_t t = blockIdx.x; t < ntiles && !abort_s; t += gridDim.x) {
        if (!mbar_wait(smem_u32(&empty[stage]), phase ^ 1)) { fail(); break; }
        const uint32_t fb = smem_u32(&full[stage]);
        mbar_expect_tx(fb, (uint32_t)SEL_TILE_BYTES);
        const uint32_t d = smem_u32(tiles + stage * SEL_TILE_BYTES);
        tma_load_2d(d, &map_db, 0, (int)(t * 128), fb);
        tma_load_2d(d + SEL_TILE_BYTES / 2, &map_db, 128, (int)(t * 128), fb);
        ++loads[stage];
        if (++stage == stages) { stage = 0; phase ^= 1; }
      }
      // every issued load lands before the CTA exits (see gemm_ws_kernel)
      if (!mbar_wait(qb, 0)) fail();
      if (abort_s) {
        for (int s2 = 0; s2 < stages; ++s2)
          if (loads[s2] > 0) mbar_wait(smem_u32(&full[s2]), (loads[s2] - 1) & 1u);
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issue
    if (lane == 0) {
      const uint32_t idesc = sel_idesc(N);
      const uint32_t qa = smem_u32(sq);
      bool any = false;
      if (!mbar_wait(smem_u32(&q_full), 0)) fail();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      int stage = 0;
      uint32_t phase = 0;
      int b = 0;
      uint32_t acc_phase = 0;
      for (int64_t t = blockIdx.x; t < ntiles && !abort_s; t += gridDim.x) {
        if (!mbar_wait(smem_u32(&acc_empty[b]), acc_phase ^ 1)) { fail(); break; }
        if (!mbar_wait(smem_u32(&full[stage]), phase)) { fail(); break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(b * N);
        const uint32_t d0 = smem_u32(tiles + stage * SEL_TILE_BYTES);
#pragma unroll
        for (int ks = 0; ks < SK / 32; ++ks) {
          const uint32_t h = (uint32_t)(ks >> 2), ko = (uint32_t)(ks & 3) * 32;
          const uint64_t da = umma_desc_sw128(d0 + h * (SEL_TILE_BYTES / 2) + ko);
          const uint64_t db = umma_desc_sw128(qa + h * (uint32_t)(N * 128) + ko);
          const uint32_t accum = ks > 0 ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n"
              :: "r"(acc), "l"(da), "l"(db), "r"(idesc), "r"(accum));
        }
        any = true;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(smem_u32(&empty[stage])) : "memory");
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(smem_u32(&acc_full[b])) : "memory");
        if (++stage == stages) { stage = 0; phase ^= 1; }
        if (++b == 2) { b = 0; acc_phase ^= 1; }
      }
      if (any) {
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(smem_u32(&mma_done)) : "memory");
        if (!mbar_wait(smem_u32(&mma_done), 0)) fail();
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int e = warp - 2;
    const int qr = warp & 3;                      // tensor-memory lanes 32qr .. 32qr + 31
    const int c_first = (e >> 2) * 16;            // 16-column groups, alternating halves
    int b = 0;
    uint32_t acc_phase = 0;
    for (int64_t t = blockIdx.x; t < ntiles && !abort_s; t += gridDim.x) {
      if (!mbar_wait(smem_u32(&acc_full[b]), acc_phase)) { if (lane == 0) fail(); break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int64_t row = t * 128 + qr * 32 + lane;
#pragma unroll 1
      for (int c0 = c_first; c0 < N; c0 += 32) {
        uint32_t v[16];
        const uint32_t taddr = tmem + ((uint32_t)(qr * 32) << 16) + (uint32_t)(b * N + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
            "%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
              "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
              "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        // the 32 lanes are 32 rows of the same query column: per column one
        // atomic reserves the slots of every lane that passes, and lane 0
        // issues the atomics of all 16 columns back to back so that their
        // latencies overlap
        unsigned m[16];
        int base[16] = {};
#pragma unroll
        for (int j = 0; j < 16; ++j)      // padding columns have tau = +inf
          m[j] = __ballot_sync(0xffffffffu, row < a.n && __uint_as_float(v[j]) >= tau_s[c0 + j]);
        if (lane == 0) {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            base[j] = m[j] ? atomicAdd(a.count + q0 + c0 + j, __popc(m[j])) : 0;
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          if (m[j] == 0) continue;                         // warp-uniform
          const int b0 = __shfl_sync(0xffffffffu, base[j], 0);
          if ((m[j] >> lane) & 1u) {
            const int q = q0 + c0 + j;
            const int slot = b0 + __popc(m[j] & ((1u << lane) - 1u));
            if (slot < a.cap) {
              a.cand[(int64_t)q * a.cap + slot] = row;
              a.cand_score[(int64_t)q * a.cap + slot] = __uint_as_float(v[j]);
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acc_empty[b]));
      if (++b == 2) { b = 0; acc_phase ^= 1; }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(tcols));
}

// Residue classes of sequences placed in the padded row layout: row
// row0[s] + i holds the class (0..19 as ARNDCQEGHILKMFPSTWYV, 20 for any
// other byte) of byte off[s] + i, i < len[s]; other rows are left as set
// by the caller (255: padding).  One block per sequence.
__global__ void layout_kernel(const uint8_t* ascii, const int64_t* off, const int32_t* len,
                              const int64_t* row0, uint8_t* cls) {
  const int s = blockIdx.x;
  const int n = len[s];
  const uint8_t* src = ascii + off[s];
  uint8_t* dst = cls + row0[s];
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = ascii_class(src[i]);
}

// Per row of x [rows][n]: the k-th largest value (k >= 1, k <= n <= 8192),
// by a bitonic sort of the row in shared memory.
constexpr int kKthMax = 8192;
__global__ void __launch_bounds__(1024) kth_largest_kernel(const float* x, int n, int k,
                                                           float* out) {
  __shared__ float v[kKthMax];
  const float* row = x + (int64_t)blockIdx.x * n;
  int size = 1;
  while (size < n) size <<= 1;
  for (int i = threadIdx.x; i < size; i += blockDim.x) v[i] = i < n ? row[i] : -INFINITY;
  __syncthreads();
  for (int len = 2; len <= size; len <<= 1) {
    for (int stride = len >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < size; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool desc = (i & len) == 0;     // descending runs first
          const float a = v[i], b = v[j];
          if (desc ? (a < b) : (a > b)) { v[i] = b; v[j] = a; }
        }
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) out[blockIdx.x] = v[k - 1];
}

int grid_for(int64_t work, int threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((work + threads - 1) / threads,
                                                    (int64_t)device_sm_count() * 16));
}

}  // namespace emb
}  // namespace sseqs

using namespace sseqs;
using namespace sseqs::emb;

static __device__ int g_tc_err;
static bool g_tc_enabled = true;

static int* tc_err_ptr() {
  static int* p[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (!p[dev]) {
    void* q = nullptr;
    if (cudaGetSymbolAddress(&q, g_tc_err) != cudaSuccess) return nullptr;
    p[dev] = static_cast<int*>(q);
  }
  return p[dev];
}

template <int EPI>
int launch_tc(const GemmArgs& g, cudaStream_t stream) {
  auto fn = gemm_tc_kernel<EPI>;
  int* err = tc_err_ptr();
  if (!err) return SSEQS_ERR_CUDA;
  if (cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)TC_SMEM) != cudaSuccess)
    return SSEQS_ERR_CUDA;
  const int64_t grid = (g.M + TC_BM - 1) / TC_BM;
  if (grid > INT32_MAX) return SSEQS_ERR_UNSUPPORTED;
  { fn<<<(unsigned)grid, TC_THREADS, TC_SMEM, stream>>>(g, err); count_launches(1); }
  return status_of(cudaGetLastError());
}

// Tensor map of a row-major bf16 array of `rows` rows of `row_len`
// elements (row stride ld elements), boxes of 64 x box_rows, 128-byte swizzle;
// rows past the end read as zero.
static bool make_map(CUtensorMap* map, const void* base, int64_t row_len, int64_t rows,
                     int64_t ld, int box_rows) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      return false;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[2] = {(cuuint64_t)row_len, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// Tensor map of `rows` FP8 codes of 256 bytes (row-major, packed), boxes of
// 128 bytes x box_rows, 128-byte swizzle; rows past the end read as zero.
static bool make_map_u8(CUtensorMap* map, const void* base, int64_t rows, int box_rows) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      return false;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[2] = {(cuuint64_t)SK, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)SK};
  const cuuint32_t box[2] = {128, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides,
                box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// The TMA-fed kernel applies when the operands' K tiles are boxes: A with
// lda >= K (a plain matrix) or lda % 64 == 0 (an overlapping row view), B
// with ldb >= K; 16-byte aligned bases and strides (checked by the caller).
static bool ws_applies(const GemmArgs& g) {
  return (g.lda >= g.K || g.lda % TC_BK == 0) && g.ldb >= g.K && g.lda <= INT32_MAX &&
         g.M + g.K / std::max<int64_t>(1, g.lda) < INT32_MAX;
}

template <int EPI>
int launch_tc_ws(const GemmArgs& g, cudaStream_t stream) {
  int* err = tc_err_ptr();
  if (!err) return SSEQS_ERR_CUDA;
  // A: lda-wide rows (the K tile at k0 is column k0 % lda of row m + k0 / lda)
  const int64_t a_len = g.lda >= g.K ? g.K : g.lda;
  const int64_t a_rows = g.M + (g.lda >= g.K ? 0 : (g.K - 1) / g.lda);
  CUtensorMap ma, mb;
  if (!make_map(&ma, g.A, a_len, a_rows, g.lda, TC_BM) ||
      !make_map(&mb, g.B, g.K, TC_BN, g.ldb, TC_BN))
    return SSEQS_ERR_CUDA;
  auto fn = gemm_ws_kernel<EPI>;
  if (cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)WS_SMEM) != cudaSuccess)
    return SSEQS_ERR_CUDA;
  const int64_t ntiles = (g.M + TC_BM - 1) / TC_BM;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, device_sm_count()));
  const int row_len = (int)(g.lda >= g.K ? (g.K + TC_BK) : g.lda);   // > every k0 when plain
  { fn<<<grid, WS_THREADS, WS_SMEM, stream>>>(ma, mb, g, row_len, err); count_launches(1); }
  return status_of(cudaGetLastError());
}

// 1 = use the tcgen05 kernel where it applies (default), 0 = mma.sync only.
extern "C" int sseqs_gemm_set_tensor_path(int tcgen05) {
  g_tc_enabled = tcgen05 != 0;
  return SSEQS_OK;
}

// Reads and clears the flag a tcgen05 GEMM sets when one of its bounded
// waits runs out (synchronises the device).
extern "C" int sseqs_gemm_error(int* out) {
  int* p = tc_err_ptr();
  if (!p || !out) return SSEQS_ERR_ARG;
  int zero = 0;
  if (cudaMemcpy(out, p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SSEQS_ERR_CUDA;
  if (cudaMemcpy(p, &zero, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return SSEQS_ERR_CUDA;
  return SSEQS_OK;
}

extern "C" int sseqs_gemm_bf16(int a_t, int b_t, int epilogue, int64_t M, int64_t N, int64_t K,
                               const void* A, int64_t lda, const void* B, int64_t ldb, void* C,
                               int64_t ldc, void* C2, const float* bias, const void* aux,
                               const uint8_t* row_mask, const void* res, cudaStream_t stream) {
  if (M < 0 || N < 0 || K < 0 || (K % BK) != 0) return SSEQS_ERR_ARG;
  if (M == 0 || N == 0) return SSEQS_OK;
  if (!A || !B || !C) return SSEQS_ERR_ARG;
  // every 16-byte chunk the tiles load must be aligned
  auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  if (!al(A) || !al(B) || (lda % 8) != 0 || (ldb % 8) != 0) return SSEQS_ERR_ARG;
  if (a_t && (M % 8) != 0) return SSEQS_ERR_ARG;
  if (b_t && (N % 8) != 0) return SSEQS_ERR_ARG;
  if (epilogue == EPI_BIAS_GELU && !bias) return SSEQS_ERR_ARG;
  if ((epilogue == EPI_GELU_GRAD || epilogue == EPI_GELU_GRAD_RES) && !aux) return SSEQS_ERR_ARG;
  if ((epilogue == EPI_BIAS_GELU_RES && (!bias || !res)) ||
      (epilogue == EPI_GELU_GRAD_RES && (!C2 || !res)))
    return SSEQS_ERR_ARG;
  if (epilogue < 0 || epilogue > 6) return SSEQS_ERR_ARG;
  GemmArgs g{M, N, K, static_cast<const __nv_bfloat16*>(A), lda,
             static_cast<const __nv_bfloat16*>(B), ldb, C, ldc,
             static_cast<__nv_bfloat16*>(C2), bias, static_cast<const __nv_bfloat16*>(aux),
             row_mask, static_cast<const __nv_bfloat16*>(res)};
  if (epilogue == EPI_F32_ADD) {
    // split K so that the grid covers every SM twice (C holds the sum of
    // the partial products; the caller zeroes it)
    if (a_t != 1 || b_t != 1) return SSEQS_ERR_UNSUPPORTED;
    const int64_t tiles = ((M + BM - 1) / BM) * ((N + BN - 1) / BN);
    const int64_t want = (2 * (int64_t)device_sm_count() + tiles - 1) / tiles;
    const int splits = (int)std::max<int64_t>(1, std::min<int64_t>(want, K / BK));
    return launch_gemm<true, true, EPI_F32_ADD>(g, stream, splits);
  }
  // N = 256, K % 64 == 0, row-major operands: the tcgen05 kernel
  if (g_tc_enabled && !a_t && !b_t && N == TC_BN && K >= TC_BK && (K % TC_BK) == 0 &&
      (ldc % 8) == 0 &&
      (reinterpret_cast<uintptr_t>(C) & 15) == 0 && (!C2 || (reinterpret_cast<uintptr_t>(C2) & 15) == 0) &&
      (!res || (reinterpret_cast<uintptr_t>(res) & 15) == 0) &&
      (!aux || (reinterpret_cast<uintptr_t>(aux) & 15) == 0) &&
      epilogue != EPI_F32 && epilogue != EPI_F32_ADD) {
    if (ws_applies(g)) {
      switch (epilogue) {
        case EPI_BF16: return launch_tc_ws<EPI_BF16>(g, stream);
        case EPI_BIAS_GELU: return launch_tc_ws<EPI_BIAS_GELU>(g, stream);
        case EPI_GELU_GRAD: return launch_tc_ws<EPI_GELU_GRAD>(g, stream);
        case EPI_BIAS_GELU_RES: return launch_tc_ws<EPI_BIAS_GELU_RES>(g, stream);
        case EPI_GELU_GRAD_RES: return launch_tc_ws<EPI_GELU_GRAD_RES>(g, stream);
      }
    }
    switch (epilogue) {
      case EPI_BF16: return launch_tc<EPI_BF16>(g, stream);
      case EPI_BIAS_GELU: return launch_tc<EPI_BIAS_GELU>(g, stream);
      case EPI_GELU_GRAD: return launch_tc<EPI_GELU_GRAD>(g, stream);
      case EPI_BIAS_GELU_RES: return launch_tc<EPI_BIAS_GELU_RES>(g, stream);
      case EPI_GELU_GRAD_RES: return launch_tc<EPI_GELU_GRAD_RES>(g, stream);
    }
  }
  if (epilogue == EPI_BIAS_GELU_RES || epilogue == EPI_GELU_GRAD_RES) {
    if (a_t || b_t) return SSEQS_ERR_UNSUPPORTED;
    return epilogue == EPI_BIAS_GELU_RES ? launch_gemm<false, false, EPI_BIAS_GELU_RES>(g, stream)
                                         : launch_gemm<false, false, EPI_GELU_GRAD_RES>(g, stream);
  }
  const int key = (a_t ? 8 : 0) | (b_t ? 4 : 0) | (epilogue & 3);
  switch (key) {
    case 0: return launch_gemm<false, false, EPI_F32>(g, stream);
    case 1: return launch_gemm<false, false, EPI_BF16>(g, stream);
    case 2: return launch_gemm<false, false, EPI_BIAS_GELU>(g, stream);
    case 3: return launch_gemm<false, false, EPI_GELU_GRAD>(g, stream);
    case 8 | 4 | 0: return launch_gemm<true, true, EPI_F32>(g, stream);
    default: return SSEQS_ERR_UNSUPPORTED;
  }
}

extern "C" int sseqs_embed_conv1_table(const uint8_t* cls, int64_t P, const float* T,
                                       const float* bias, const uint8_t* row_mask, int D,
                                       void* Y, void* Z, cudaStream_t stream) {
  if (P < 0 || D <= 0 || D % 8 != 0 || D > 512) return SSEQS_ERR_ARG;
  if (P == 0) return SSEQS_OK;
  if (!cls || !T || !bias || !Y) return SSEQS_ERR_ARG;
  auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  if (!al(T) || !al(Y) || (Z && !al(Z))) return SSEQS_ERR_ARG;
  const size_t smem = sizeof(float) * 5 * 21 * (size_t)D;
  if (cudaFuncSetAttribute((const void*)conv1_table_kernel,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return SSEQS_ERR_CUDA;
  const int64_t work = P * (D / 8);
  const int grid = (int)std::max<int64_t>(
      1, std::min<int64_t>((work + 255) / 256, (int64_t)device_sm_count() * 4));
  { conv1_table_kernel<<<grid, 256, smem, stream>>>(
        cls, P, T, bias, row_mask, D, static_cast<__nv_bfloat16*>(Y),
        static_cast<__nv_bfloat16*>(Z));
    count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_embed_lookup(const uint8_t* cls, int64_t P, const void* E, int D, void* X,
                                  cudaStream_t stream) {
  if (P < 0 || D <= 0 || (P > 0 && (!cls || !E || !X))) return SSEQS_ERR_ARG;
  if (P == 0) return SSEQS_OK;
  { embed_lookup_kernel<<<grid_for(P * D, 256), 256, 0, stream>>>(
        cls, P, static_cast<const __nv_bfloat16*>(E), D, static_cast<__nv_bfloat16*>(X));
    count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_embed_grad(const uint8_t* cls, int64_t P, const void* dX, int D, float* dE,
                                cudaStream_t stream) {
  if (P < 0 || D <= 0 || (P > 0 && (!cls || !dX || !dE))) return SSEQS_ERR_ARG;
  if (P == 0) return SSEQS_OK;
  { embed_grad_kernel<<<grid_for(P * D, 256), 256, 0, stream>>>(
        cls, P, static_cast<const __nv_bfloat16*>(dX), D, dE);
    count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_pool_normalize(const void* Y, int D, const int64_t* start, const int32_t* len,
                                    int n_seqs, float* pooled, float* emb, float* inv_norm,
                                    cudaStream_t stream) {
  if (n_seqs < 0 || D < 32 || D > 1024 || (D % 32) != 0) return SSEQS_ERR_ARG;
  if (n_seqs == 0) return SSEQS_OK;
  if (!Y || !start || !len || !pooled || !emb || !inv_norm) return SSEQS_ERR_ARG;
  { pool_normalize_kernel<<<n_seqs, D, 0, stream>>>(static_cast<const __nv_bfloat16*>(Y), start,
                                                    len, pooled, emb, inv_norm);
    count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_pair_loss(const float* emb, int D, const int32_t* ia, const int32_t* ib,
                               const float* y, const float* weight, int64_t B, float* dE,
                               float* loss, float* pred, cudaStream_t stream) {
  if (B < 0 || D <= 0 || (B > 0 && (!emb || !ia || !ib || !y || !loss))) return SSEQS_ERR_ARG;
  if (B == 0) return SSEQS_OK;
  const int64_t threads = B * 32;
  const int grid = (int)((threads + 255) / 256);
  { pair_loss_kernel<<<grid, 256, 0, stream>>>(emb, D, ia, ib, y, weight, B, dE, loss, pred);
    count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_pool_backward(const float* emb, const float* dE, const float* inv_norm,
                                   const int64_t* start, const int32_t* len, int n_seqs, int D,
                                   const void* Z, void* dZ, void* G, cudaStream_t stream) {
  if (n_seqs < 0 || D < 32 || D > 1024 || (D % 32) != 0) return SSEQS_ERR_ARG;
  if (n_seqs == 0) return SSEQS_OK;
  if (!emb || !dE || !inv_norm || !start || !len || !Z || !dZ) return SSEQS_ERR_ARG;
  { pool_backward_kernel<<<n_seqs, D, 0, stream>>>(emb, dE, inv_norm, start, len,
                                                   static_cast<const __nv_bfloat16*>(Z),
                                                   static_cast<__nv_bfloat16*>(dZ),
                                                   static_cast<__nv_bfloat16*>(G));
    count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_bias_grad(const void* dZ, int64_t P, int D, float* db, cudaStream_t stream) {
  if (P < 0 || D <= 0 || (P > 0 && (!dZ || !db))) return SSEQS_ERR_ARG;
  if (P == 0) return SSEQS_OK;
  const int chunks = (int)std::min<int64_t>(P, (int64_t)device_sm_count() * 4);
  const dim3 grid(chunks, (D + 255) / 256);
  { bias_grad_kernel<<<grid, 256, 0, stream>>>(static_cast<const __nv_bfloat16*>(dZ), P, D, db);
    count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_adam_conv(float* w, float* m, float* v, const float* dWT, int Cout, int Cin,
                               float lr, float b1, float b2, float eps, int step, void* Wb,
                               void* Wf, cudaStream_t stream) {
  if (Cout <= 0 || Cin <= 0 || step < 1 || !w || !m || !v || !dWT || !Wb || !Wf)
    return SSEQS_ERR_ARG;
  AdamArgs o{lr, b1, b2, eps, 1.f - powf(b1, (float)step), 1.f - powf(b2, (float)step)};
  { adam_conv_kernel<<<grid_for((int64_t)Cout * 5 * Cin, 256), 256, 0, stream>>>(
        w, m, v, dWT, Cout, Cin, o, static_cast<__nv_bfloat16*>(Wb),
        static_cast<__nv_bfloat16*>(Wf));
    count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_adam_flat(float* w, float* m, float* v, const float* g, int64_t n, float lr,
                               float b1, float b2, float eps, int step, void* wb,
                               cudaStream_t stream) {
  if (n < 0 || step < 1 || (n > 0 && (!w || !m || !v || !g))) return SSEQS_ERR_ARG;
  if (n == 0) return SSEQS_OK;
  AdamArgs o{lr, b1, b2, eps, 1.f - powf(b1, (float)step), 1.f - powf(b2, (float)step)};
  { adam_flat_kernel<<<grid_for(n, 256), 256, 0, stream>>>(w, m, v, g, n, o,
                                                          static_cast<__nv_bfloat16*>(wb));
    count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_quantize_e4m3(const float* x, int64_t n, float scale, uint8_t* out,
                                   cudaStream_t stream) {
  if (n < 0 || (n > 0 && (!x || !out))) return SSEQS_ERR_ARG;
  if (n == 0) return SSEQS_OK;
  { quantize_e4m3_kernel<<<grid_for(n, 256), 256, 0, stream>>>(x, n, scale, out);
    count_launches(1); }
  return status_of(cudaGetLastError());
}

static size_t score_smem(int stages) { return (size_t)(1 + stages) * 128 * SLD; }

extern "C" int sseqs_score_select(const uint8_t* Q, int nq, const uint8_t* DB, int64_t n,
                                  const float* tau, int32_t* count, int64_t* cand,
                                  float* cand_score, int cap, cudaStream_t stream) {
  if (nq < 0 || n < 0 || cap < 0) return SSEQS_ERR_ARG;
  if (nq == 0 || n == 0) return SSEQS_OK;
  if (!Q || !DB || !tau || !count || !cand || !cand_score) return SSEQS_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(Q) & 15) || (reinterpret_cast<uintptr_t>(DB) & 15))
    return SSEQS_ERR_ARG;
  SelArgs a{Q, nq, DB, n, tau, count, cand, cand_score, cap};
  if (g_tc_enabled && n < (int64_t)INT32_MAX - 256) {
    // tcgen05: query tiles of N = the batch rounded up to 16 (at most 256)
    int* err = tc_err_ptr();
    if (!err) return SSEQS_ERR_CUDA;
    const int N = std::min(256, (nq + 15) / 16 * 16);
    const int qt = (nq + N - 1) / N;
    const int stages = (int)std::min<int64_t>(
        SEL_STAGES_MAX, (227 * 1024 - 4096 - (int64_t)N * SK) / SEL_TILE_BYTES);
    const size_t smem = (size_t)N * SK + (size_t)stages * SEL_TILE_BYTES + 1024;
    CUtensorMap mdb, mq;
    if (!make_map_u8(&mdb, DB, n, 128) || !make_map_u8(&mq, Q, nq, N)) return SSEQS_ERR_CUDA;
    if (cudaFuncSetAttribute((const void*)score_select_tc_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return SSEQS_ERR_CUDA;
    const int64_t ntiles = (n + 127) / 128;
    const int per_tile = std::max(1, device_sm_count() / qt);
    const int gx = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, per_tile));
    { score_select_tc_kernel<<<dim3(gx, qt), SEL_THREADS, smem, stream>>>(mdb, mq, a, N, stages,
                                                                            err);
      count_launches(1); }
    return status_of(cudaGetLastError());
  }
  const size_t smem = score_smem(2);
  if (cudaFuncSetAttribute((const void*)score_select_kernel,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return SSEQS_ERR_CUDA;
  const int qt = (nq + 127) / 128;
  const int64_t ntiles = (n + 127) / 128;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, score_select_kernel, GEMM_THREADS, smem) !=
          cudaSuccess || nb < 1)
    return SSEQS_ERR_CUDA;
  const int64_t slots = (int64_t)device_sm_count() * nb;
  const int gx = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (slots + qt - 1) / qt));
  { score_select_kernel<<<dim3(gx, qt), GEMM_THREADS, smem, stream>>>(a); count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_score_dense(const uint8_t* Q, int nq, const uint8_t* DB, int64_t n,
                                 float* out, cudaStream_t stream) {
  if (nq < 0 || n < 0) return SSEQS_ERR_ARG;
  if (nq == 0 || n == 0) return SSEQS_OK;
  if (!Q || !DB || !out) return SSEQS_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(Q) & 15) || (reinterpret_cast<uintptr_t>(DB) & 15))
    return SSEQS_ERR_ARG;
  SelArgs a{Q, nq, DB, n, nullptr, nullptr, nullptr, nullptr, 0};
  const size_t smem = score_smem(1);
  if (cudaFuncSetAttribute((const void*)score_dense_kernel,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return SSEQS_ERR_CUDA;
  const int64_t gx = (n + 127) / 128;
  if (gx > INT32_MAX) return SSEQS_ERR_UNSUPPORTED;
  { score_dense_kernel<<<dim3((unsigned)gx, (nq + 127) / 128), GEMM_THREADS, smem, stream>>>(a, out);
    count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_embed_layout(const uint8_t* ascii, const int64_t* off, const int32_t* len,
                                  const int64_t* row0, int n_seqs, uint8_t* cls,
                                  cudaStream_t stream) {
  if (n_seqs < 0 || (n_seqs > 0 && (!ascii || !off || !len || !row0 || !cls)))
    return SSEQS_ERR_ARG;
  if (n_seqs == 0) return SSEQS_OK;
  { layout_kernel<<<n_seqs, 128, 0, stream>>>(ascii, off, len, row0, cls); count_launches(1); }
  return status_of(cudaGetLastError());
}

extern "C" int sseqs_kth_largest_rows(const float* x, int rows, int n, int k, float* out,
                                      cudaStream_t stream) {
  if (rows < 0 || n < 1 || n > kKthMax || k < 1 || k > n) return SSEQS_ERR_ARG;
  if (rows == 0) return SSEQS_OK;
  if (!x || !out) return SSEQS_ERR_ARG;
  { kth_largest_kernel<<<rows, 1024, 0, stream>>>(x, n, k, out); count_launches(1); }
  return status_of(cudaGetLastError());
}
