// Score-only Smith-Waterman kernel template (linear and affine gaps), sm_100a.
//
// Semantics are those of the reference kernels sseqs/sw.cu:55-179 (linear)
// and sseqs/sw.cu:182-325 (affine): the query is cut into 32 stripes of
// TPT = ceil(Lq/32) columns; inside a row the horizontal dependency restarts
// at the first column of every stripe (H(i, j-1) := 0 there), while the
// diagonal dependency crosses stripes.  Because the rows of all stripes are
// independent of each other inside one row, the stripes can be evaluated in
// any lane mapping.
//
// B200 mapping.  Two stripes of the same target share one 32-bit register as
// int16x2: the lo halves carry stripes 0..15 and the hi halves stripes
// 16..31 (word w of lane gl: stripes gl*W + w and 16 + gl*W + w).  A lane
// holds W such words per column, so a target occupies G = 32/(2W) lanes and
// a warp scores 2W targets side by side.  With this order a word's diagonal
// input at its first column is the last column of the word before it, both
// halves at once; only the first word of a lane takes it from the lane
// before, and at lane 0 its hi half continues stripe 15 (the lo half of the
// group's last lane) while its lo half is column -1 -- one shuffle and one
// byte permute per row.  The query profile (score of each residue class
// against every column, already packed as the lane's int16x2 words) sits in
// shared memory; a lane fetches its row of it with 128-bit loads.
//
// Every int16x2 instruction used here issues at half rate on its pipe: the
// max-type DPX instructions (__vimax3_s16x2_relu, __viaddmax_s16x2_relu) on
// the ALU pipe, the int16x2 add/sub (__vadd2, __vsub2) on the FMA pipe.  A
// scheduler issues one instruction per clock, so the recurrences are written
// to spread work over both pipes:
//   affine, per word-column (2 cells): M' = D_diag + s, Mo = M' - open (FMA);
//     Ix = max(Ix_left - ext, Mo_left, 0), D = max(M', Ix, Iy, 0),
//     next-row Iy = max(Iy - ext, Mo, 0), half a running max (ALU)
//     -> 3.5 ALU + 2 FMA;
//   linear, with the state carried as H + gap: u = Hg_diag + (s - gap) (FMA),
//     H = max(u, Hg_up, Hg_left, 0), half a running max (ALU),
//     Hg = H + gap (FMA)  -> 1.5 ALU + 2 FMA.
// M' is left unclamped: it only enters maxima that also hold 0.  All cell
// values are >= 0 and at most 11 * Lq <= 22528, so int16 lanes cannot
// overflow for Lq <= 2048 (no int32 re-run is ever needed); the profile's
// padding words (-32768 + open, or -16384) keep every intermediate inside
// int16 and can never raise a score.
//
// Targets are streamed: each lane group takes targets from a launch-wide
// counter (a few at a time, the next grab issued one chunk ahead so its
// latency is hidden), which keeps every group busy until the last targets
// whatever their lengths.  A target is read R rows at a time (4, 8 or 16,
// see rows_per_fetch), the R bytes of the next step prefetched (one byte per
// lane, or R/4 + 1 aligned words per lane in groups of fewer than R lanes);
// when a target ends (rows past its end are padding rows) the
// group writes its score, resets its state and moves on while the other
// groups of the warp keep going.
#pragma once
#include <algorithm>
#include <utility>

#include "common.cuh"

namespace sseqs {
namespace sw {

constexpr int kMaxQuery = 2048;
// Target rows per byte fetch: the per-fetch bookkeeping is shared by this
// many rows, and a target's last fetch pads with up to R-1 rows.  Measured
// (300k targets): affine 8 rows beat 4 by 10% at 27 words per lane, and 16
// beat 8 by 2-3% at 16 words or fewer but lost 9% at 27 (larger code and
// register footprint; with the classes spread over the group's lanes, 16
// still lost 1-8% at widths 20-32).  Linear 8 rows beat 4 by 4-7% in the
// narrow layout up to width 13 and the wide one from 17 to 29 (one class
// register per lane); elsewhere they spill under the register caps, so
// linear keeps 4 there.  The fused kernel: 8 rows beat 4 by 1-5% in the
// narrow layout and lost 16% in the wide one (fewer blocks); they fit the
// register caps without spilling at widths 9-13 and 18-21 only.
template <int MODE, int TPT, int W>
__host__ __device__ constexpr int rows_per_fetch() {
  return (MODE == 1 || MODE == 3) ? (W * TPT <= 16 ? 16 : 8)
       : MODE == 0 && ((W == 1 && TPT <= 13) || (W == 2 && TPT > 16)) ? 8
       : MODE == 2 && W == 1 && (TPT <= 13 || (TPT >= 18 && TPT <= 21)) ? 8 : 4;
}

struct SwArgs {
  const uint8_t* q;       // query residue classes
  int Lq;
  const int32_t* idx;     // target -> window index g (nullable: g = g0 + t)
  int32_t g0;
  int64_t n;              // number of targets
  const uint8_t* ascii;   // target bytes
  const int32_t* starts;  // window table (reference semantics)
  int skip;               // bytes not scored at the start of every window
  int32_t* out;
  int p0, p1;             // linear: gap; affine: open, extend; both: gap, open
  unsigned int* ticket;   // zeroed launch-wide target counter (fast kernel)
  int chunk;              // targets per counter grab (fast kernel, >= 1)
  int p2;                 // both: extend
  int32_t* out2;          // both: affine scores (out: linear)
  int skip2;              // both: the affine windows start this many (0 or 1)
                          // bytes after the linear ones
};

// Several queries of the same stripe width in one launch: blockIdx.y picks
// the query, which reads lens[y] (device) residues at q + y * q_stride,
// scores the targets idx + y * idx_stride (when idx is given), writes its
// scores at out + y * out_stride and takes targets from ticket[y].  n == 0
// is the single-query launch (SwArgs alone).  A length
// that does not belong to the launch's stripe width (or exceeds q_stride)
// is not scored: its output row is filled with INT32_MIN.
constexpr int kMaxLaunchQueries = 128;
struct QueryTable {
  const int32_t* lens;
  int64_t out_stride;
  int64_t idx_stride;
  int32_t q_stride;
  int32_t n;
};

// Window of one target (sseqs/sw.cu:66-77): rows [pos, end), or no rows and
// an immediate result (-1 for an empty or inverted window, 0 otherwise).
// Window bounds come from int32 delimiter positions, so rows with bytes lie
// in [0, 2^31) and fit 32-bit arithmetic.
struct Win {
  uint32_t pos, end;
  int32_t res;
  bool rows;
};

__device__ __forceinline__ Win window_of(const SwArgs& a, int64_t t) {
  const int32_t g = a.idx ? a.idx[t] : (int32_t)(a.g0 + t);
  const int64_t base = (g == 0) ? -1 : (int64_t)a.starts[g - 1];
  const int64_t len = (int64_t)a.starts[g] - base - 1;
  const int64_t pos = base + 1 + a.skip, end = base + 1 + len;
  Win w;
  w.pos = (uint32_t)pos;
  w.end = (uint32_t)end;
  if (len == 0 || len < -1) {
    w.rows = false;
    w.res = -1;
  } else {
    w.rows = pos < end;
    w.res = 0;
  }
  return w;
}

__device__ __forceinline__ int score_of(const uint8_t* q, int Lq, int cls, int j) {
  if (j >= Lq || cls == kClsPad) return kNeg;
  if (cls >= kNumAA) return -4;
  const int qc = q[j];
  return qc < kNumAA ? blosum62(cls, qc) : -4;
}

// Words per lane for a stripe width: the narrow variant keeps a target on
// 16 lanes down to TPT 9 and widens below; the wide variant gives each lane
// twice the columns (fewer lanes per target, more targets per warp) for
// TPT <= 16, and for the linear kernel up to TPT 29 (two independent
// recurrence chains per lane; measured on B200 it beat the narrow layout by
// 7-11% at widths 20-27, where the linear kernel waits on the latency of
// its one chain; the affine kernel, bound by its ALU pipe, lost 1-20%).
// Wide equals narrow where no wide layout exists.  The choice per width is
// made by the autotuner at run time.
template <int TPT, bool WIDE, int MODE>
constexpr int words_for() {
  if (WIDE && MODE == 0 && TPT > 16 && TPT <= 29) return 2;
  if (WIDE) return TPT == 1 ? 16 : TPT == 2 ? 16 : TPT <= 4 ? 8 : TPT <= 8 ? 4 : TPT <= 16 ? 2 : 1;
  return TPT == 1 ? 16 : TPT == 2 ? 8 : TPT <= 4 ? 4 : TPT <= 8 ? 2 : 1;
}

// Profile layout of one residue class.  Lane-major: lane gl's NV 16-byte
// vectors are contiguous, padded to an odd count so that the 8 lanes of a
// quarter warp hit distinct banks.  Vector-major (VM): vector v of lane gl
// at slot v * G + gl, so those 8 lanes read 8 consecutive slots (all 32
// banks once) with no padding -- up to 25% less shared memory, which gave
// the fused kernel a third block per SM at widths 21-24 (3.5-6.6% faster)
// and the wide linear layout at 27 2.6% faster; with fewer than 16 lanes
// per target it was 1-3% slower elsewhere (the quarter warp then spans
// groups reading different classes), so those keep the lane-major layout
// (the wide linear layout takes VM from width 19).
template <int TPT, int W, int MODE>
constexpr bool vector_major() { return W == 1 || (MODE == 0 && W == 2 && TPT > 18); }

template <int TPT, int W, bool VM, bool PAIR = false>
struct Layout {
  // lanes per target: a lane holds 2W stripes (two per word), or W stripes
  // of two queries in the query-pair mode
  static constexpr int G = PAIR ? 32 / W : 32 / (2 * W);
  static constexpr int GPW = 32 / G;        // targets per warp
  static constexpr int NWD = W * TPT;       // profile words per lane and row
  static constexpr int NV = (NWD + 3) / 4;  // 128-bit loads per lane and row
  static constexpr int LWP = VM ? NV * 4 : ((NV % 2) ? NV : NV + 1) * 4;  // words per lane
  static constexpr int CLS = G * LWP;       // words per residue class
  static constexpr int LANE_STEP = VM ? 1 : LWP / 4;   // uint4 slots from lane to lane
  static constexpr int VEC_STEP = VM ? G : 1;          // uint4 slots from vector to vector
  static constexpr size_t smem = (size_t)kNumCls * CLS * 4 + 256;
};

// The linear recurrence issues 2 int16x2 adds per word on the FMA pipe
// (both half rate) and 1.5 maxima on the ALU pipe, so its FMA pipe is the
// busier one (ncu at width 27: 2.4 FMA against 1.9 ALU instructions per
// word).  Every kLinAluEvery-th column takes the add onto the ALU pipe
// (one add-max instead of add + max); measured on B200 (300k targets, same
// scores) every 4th column was 0.3-3% faster at widths 13-32 and 2% slower
// at width 5 (every 2nd or 3rd: mixed, -3% to +1%), so it applies from
// width 9 -- except 17-18, where it made the wide layout spill.
template <int TPT>
constexpr int lin_alu_every() { return TPT >= 9 && (TPT < 17 || TPT > 18) ? 4 : 0; }

// Score variants of one instantiation: the linear kernel, the affine kernel,
// or both in one pass over the targets (the exact search scores every
// target with both; one pass shares the byte fetch, the per-row loads and
// the bookkeeping, and lets the linear recurrence -- FMA-pipe heavy -- fill
// the ALU pipe slack the affine one leaves, and vice versa).
constexpr int kLin = 0, kAff = 1, kBoth = 2;
// Query-pair mode: the affine recurrence of two queries of the same stripe
// width against the same targets, the lo half of every word holding stripe m
// of query A and the hi half stripe m of query B.  The two share the byte
// fetch, the class of every row, the profile-row load and the bookkeeping;
// and since both halves of a word belong to the same stripe, the diagonal
// input of a stripe's first column is simply the previous word (no byte
// permute across halves).
constexpr int kPair = 3;
constexpr int kModes = 4;

// Block shape per instantiation.  The state of a lane is about NWD words
// (linear: H; affine: D and Iy; both: all three) plus its profile rows, so
// registers grow with NWD.  Up to ~128 registers a block has 8 warps that
// share one copy of the query profile in shared memory, with the register
// cap set for 3 blocks (85 registers) or 2 (128) per SM; larger states use
// blocks of 4 warps, which pack the register file more finely (the fused
// kernel and the wide linear layout capped for 3 of them, 170 registers,
// when the estimate allows).  The affine kernel at 17 words per lane (8
// rows per fetch) ran 7% slower under the 85-register cap than with 128, so
// the 3-block cap is not used where affine fetches 8 rows.
template <int TPT, int W, int MODE>
struct Shape {
  static constexpr int NWD = W * TPT;
  static constexpr int est_regs = (MODE == kAff || MODE == kPair) ? 3 * NWD + 32
                                : MODE == kLin ? 2 * NWD + 53 : 5 * NWD + 40;
  // (the query-pair kernel carries query B's row and flags besides: it
  // spilled under the 85-register cap at 12 and 16 words per lane, so it
  // takes the cap up to 10)
  static constexpr bool cap85 = est_regs <= 85 && (MODE != kPair || NWD <= 10) &&
                                !(MODE == kAff && rows_per_fetch<MODE, TPT, W>() == 8);
  static constexpr int threads = est_regs <= 128 ? 256 : 128;
  static constexpr int min_blocks =
      threads == 256 ? (cap85 ? 3 : 2)
                     : ((MODE == kBoth || (MODE == kLin && TPT > 16 && W == 2)) &&
                        est_regs <= 170 ? 3 : 1);
};

// The gap parameters msa() always passes (sseqs/msa.py:317, 331-332):
// linear gap -1, affine open 11 and extend 1.  Every kernel has a twin
// (DEF = true) with these as compile-time constants, picked by the host
// whenever a call passes them; the int16x2 gap words then reach the DPX
// instructions as immediates instead of registers.  Measured on B200 (1M
// segments, widths 2-32): the affine kernel 5-16% faster (8% at most
// widths) with scores unchanged; gap words passed as pre-packed kernel
// parameters instead were 0-7% slower.
constexpr int kDefGap = -1, kDefOpen = 11, kDefExt = 1;

template <int TPT, int W, int MODE, bool DEF>
__global__ void __launch_bounds__(Shape<TPT, W, MODE>::threads, Shape<TPT, W, MODE>::min_blocks)
    sw_stream_kernel(SwArgs a, const QueryTable qt) {
  constexpr bool PAIR = MODE == kPair;
  constexpr bool VM = vector_major<TPT, W, MODE>();
  using L = Layout<TPT, W, VM, PAIR>;
  constexpr bool DO_LIN = MODE == kLin || MODE == kBoth, DO_AFF = MODE != kLin;
  constexpr int NTAB = MODE == kBoth ? 2 : 1;
  // query-pair mode: query B's residues, length and output row
  const uint8_t* qB = nullptr;
  int LqB = 0;
  int32_t* outB = nullptr;
  bool writeA = true, writeB = false;
  if constexpr (PAIR) {
    // blockIdx.y picks the pair (queries 2y and 2y + 1 of the table); a
    // query whose length does not belong to this width is not scored (its
    // row is filled with INT32_MIN) and its half runs on padding
    const int y = blockIdx.y, ia = 2 * y, ib = 2 * y + 1;
    const bool hasB = ib < qt.n;
    const int lenA = qt.lens[ia], lenB = hasB ? qt.lens[ib] : 0;
    const bool okA = lenA >= 1 && (lenA + 31) / 32 == TPT && lenA <= qt.q_stride;
    const bool okB = hasB && lenB >= 1 && (lenB + 31) / 32 == TPT && lenB <= qt.q_stride;
    a.q += (size_t)ia * qt.q_stride;
    qB = a.q + qt.q_stride;
    a.out += (int64_t)ia * qt.out_stride;
    outB = a.out + qt.out_stride;
    a.ticket += y;
    if (!okA || (hasB && !okB)) {
      for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
           i += (int64_t)gridDim.x * blockDim.x) {
        if (!okA) a.out[i] = INT32_MIN;
        if (hasB && !okB) outB[i] = INT32_MIN;
      }
    }
    if (!okA && !okB) return;
    writeA = okA;
    writeB = okB;
    a.Lq = okA ? lenA : 0;
    LqB = okB ? lenB : 0;
  } else if (qt.n > 0) {
    const int y = blockIdx.y;
    const int len = qt.lens[y];
    a.q += (size_t)y * qt.q_stride;
    a.out += (int64_t)y * qt.out_stride;
    if constexpr (MODE == kBoth) a.out2 += (int64_t)y * qt.out_stride;
    if (a.idx) a.idx += (int64_t)y * qt.idx_stride;
    a.ticket += y;
    if (len < 1 || (len + 31) / 32 != TPT || len > qt.q_stride) {
      for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
           i += (int64_t)gridDim.x * blockDim.x) {
        a.out[i] = INT32_MIN;
        if constexpr (MODE == kBoth) a.out2[i] = INT32_MIN;
      }
      return;
    }
    a.Lq = len;
  }
  constexpr int G = L::G;
  extern __shared__ uint4 smem4[];
  uint32_t* prof = reinterpret_cast<uint32_t*>(smem4);       // linear table first when both
  uint8_t* lut = reinterpret_cast<uint8_t*>(prof + NTAB * kNumCls * L::CLS);

  // Gap parameters: linear gap (p0); affine open and extend (p0, p1 in the
  // affine kernel; p1, p2 in the fused one); constants in the DEF twin.
  const int gap = DEF ? kDefGap : a.p0;
  constexpr bool AFF_ONLY = MODE == kAff || MODE == kPair;   // affine gaps in p0, p1
  const int open = DEF ? kDefOpen : AFF_ONLY ? a.p0 : a.p1;
  const int ext = DEF ? kDefExt : AFF_ONLY ? a.p1 : a.p2;

  // Profile words.  Affine: s (real columns), -32768 + open (padding), so
  // that M' - open never leaves int16.  Linear: s - gap (the state carries
  // H + gap), -16384 for padding.  Padding never raises a score.
  for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = ascii_class((uint8_t)i);
  for (int i = threadIdx.x; i < NTAB * kNumCls * L::CLS; i += blockDim.x) {
    const int tb = i / (kNumCls * L::CLS), ii = i - tb * (kNumCls * L::CLS);
    const bool aff_tab = AFF_ONLY || tb == 1;
    const int pad = aff_tab ? kNeg + open : -16384;
    const int c = ii / L::CLS, r = ii - c * L::CLS;
    const int slot = r >> 2;                          // uint4 slot in the class
    const int gl = VM ? slot % G : slot / L::LANE_STEP;
    const int v = (VM ? slot / G : slot % L::LANE_STEP) * 4 + (r & 3);   // word of lane gl
    uint32_t word = pack2(pad, pad);
    if (PAIR && v < L::NWD) {
      // stripe m = gl * W + w of query A (lo) and query B (hi)
      const int w = v / TPT, k = v - w * TPT;
      const int j = (gl * W + w) * TPT + k;
      int s0 = score_of(a.q, a.Lq, c, j), s1 = score_of(qB, LqB, c, j);
      s0 = (s0 == kNeg) ? pad : s0;
      s1 = (s1 == kNeg) ? pad : s1;
      word = pack2(s0, s1);
    } else if (v < L::NWD) {
      const int w = v / TPT, k = v - w * TPT;
      const int j = (gl * W + w) * TPT + k;             // stripe gl * W + w (lo), + 16 (hi)
      int s0 = score_of(a.q, a.Lq, c, j), s1 = score_of(a.q, a.Lq, c, j + 16 * TPT);
      s0 = (s0 == kNeg) ? pad : (aff_tab ? s0 : s0 - gap);
      s1 = (s1 == kNeg) ? pad : (aff_tab ? s1 : s1 - gap);
      word = pack2(s0, s1);
    }
    prof[i] = word;
  }
  __syncthreads();
  const uint32_t* profL = prof;
  const uint32_t* profA = prof + (MODE == kBoth ? kNumCls * L::CLS : 0);

  const int lane = threadIdx.x & 31;
  const int grp = lane / G;
  const int gl = lane - grp * G;
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (grp * G));
  const int leader = grp * G;
  // diagonal input of a lane's first word: the lane before it (rotating
  // inside the group); at lane 0 the lo half is column -1 instead
  const int src_left = (gl + G - 1) % G;
  const uint32_t sel_left = gl == 0 ? 0x1054u : 0x3210u;

  const uint32_t gap2 = pack2(gap, gap);       // linear gap, -16384 <= gap <= 0
  const uint32_t nopen2 = pack2(-open, -open); // affine -open, 0 <= open <= 16384
  const uint32_t next2 = pack2(-ext, -ext);    // affine -extend, 0 <= extend <= 16384
  // state at row -1: H = 0 (linear state is H + gap), D = Iy = 0 (affine)

  constexpr int WL = DO_LIN ? W : 1, WA = DO_AFF ? W : 1;
  uint32_t SL[WL][TPT];               // linear: H(i-1,.) + gap
  uint32_t SA[WA][TPT];               // affine: D(i-1,.)
  uint32_t Y[WA][TPT];                // affine: Iy(i,.) carried into row i
  uint32_t bestL = 0, bestA = 0;
  auto reset = [&]() {
    bestL = 0;
    bestA = 0;
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
      for (int k = 0; k < TPT; ++k) {
        if constexpr (DO_LIN) SL[w][k] = gap2;
        if constexpr (DO_AFF) { SA[w][k] = 0; Y[w][k] = 0; }
      }
  };
  reset();

  // one linear DP row for every group of the warp (warp-uniform)
  auto row_lin = [&](int cls) {
    const uint4* pr = reinterpret_cast<const uint4*>(profL + cls * L::CLS) + gl * L::LANE_STEP;
    uint32_t s[L::NV * 4];
#pragma unroll
    for (int v = 0; v < L::NV; ++v) {
      const uint4 x = pr[v * L::VEC_STEP];
      s[4 * v] = x.x; s[4 * v + 1] = x.y; s[4 * v + 2] = x.z; s[4 * v + 3] = x.w;
    }
    uint32_t din[WL];                               // diagonals, from the previous row
    din[0] = __byte_perm(__shfl_sync(0xffffffffu, SL[WL - 1][TPT - 1], src_left, G), gap2,
                         sel_left);                 // column -1 of stripe 0: H + gap = gap
#pragma unroll
    for (int w = 1; w < WL; ++w) din[w] = SL[w - 1][TPT - 1];
    uint32_t pend = 0;
#pragma unroll
    for (int w = 0; w < WL; ++w) {
      const uint32_t diag = din[w];
      // state Hg = H + gap:  H = max(Hg_diag + (s - gap), Hg_up, Hg_left, 0)
      // (Hg_left = gap at the first column of a stripe).  The next column's
      // diagonal sum is formed before S[k] is overwritten, so the new value
      // can take the old one's register.
      //
      // The running maximum is taken over the diagonal sums u rather than
      // over H: with gap <= 0 a cell whose H comes from Hg_up or Hg_left is
      // never above the cell it came from, so following those moves back
      // ends at a cell whose H is its u (or 0), and max H = max(0, max u).
      // (Padding u lie 16384 below a real cell and never win.)  Taking the
      // maximum over u keeps u a value of its own, so the compiler leaves
      // its add on the FMA pipe instead of folding it into an add-max on the
      // ALU pipe, which is the busier one.
      uint32_t hg_left = 0;
      uint32_t u = __vadd2(diag, s[w * TPT]);                               // FMA pipe
#pragma unroll
      for (int k = 0; k < TPT; ++k) {
        const uint32_t up = SL[w][k];
        const uint32_t u_next = (k + 1 < TPT) ? __vadd2(up, s[w * TPT + k + 1]) : 0u;
        constexpr int EV = lin_alu_every<TPT>();
        if (MODE == kLin && EV > 0 && k % (EV > 0 ? EV : 1) == EV - 1) {
          // the same value with the add on the ALU pipe:
          // max(m + gap, gap) = max(m, 0) + gap, m >= Hg_up >= gap >= -16384
          const uint32_t m = (k == 0) ? __vmaxs2(u, up) : __vimax3_s16x2(u, up, hg_left);
          hg_left = __viaddmax_s16x2(m, gap2, gap2);                        // ALU pipe
        } else {
          const uint32_t h = (k == 0) ? __vimax_s16x2_relu(u, up)
                                      : __vimax3_s16x2_relu(u, up, hg_left); // ALU pipe
          hg_left = __vadd2(h, gap2);                                       // FMA pipe
        }
        SL[w][k] = hg_left;
        if (((w * TPT + k) & 1) == 0) pend = u;
        else bestL = __vimax3_s16x2(bestL, pend, u);
        u = u_next;
      }
    }
    if ((L::NWD & 1) != 0) bestL = __vimax_s16x2_relu(bestL, pend);
  };

  // one affine DP row for every group of the warp (warp-uniform)
  auto row_aff = [&](int cls) {
    const uint4* pr = reinterpret_cast<const uint4*>(profA + cls * L::CLS) + gl * L::LANE_STEP;
    uint32_t s[L::NV * 4];
#pragma unroll
    for (int v = 0; v < L::NV; ++v) {
      const uint4 x = pr[v * L::VEC_STEP];
      s[4 * v] = x.x; s[4 * v + 1] = x.y; s[4 * v + 2] = x.z; s[4 * v + 3] = x.w;
    }
    uint32_t din[WA];                               // diagonals, from the previous row
    if constexpr (PAIR) {
      // both halves hold stripe gl * W + w: the lane before, 0 at lane 0
      uint32_t from_left = __shfl_up_sync(0xffffffffu, SA[WA - 1][TPT - 1], 1, G);
      if (gl == 0) from_left = 0u;                  // column -1 of stripe 0
      din[0] = from_left;
    } else {
      din[0] = __byte_perm(__shfl_sync(0xffffffffu, SA[WA - 1][TPT - 1], src_left, G), 0u,
                           sel_left);               // column -1 of stripe 0: D = 0
    }
#pragma unroll
    for (int w = 1; w < WA; ++w) din[w] = SA[w - 1][TPT - 1];
    uint32_t pend = 0;
#pragma unroll
    for (int w = 0; w < WA; ++w) {
      const uint32_t diag = din[w];
      // M' = D_diag + s (unclamped), Mo = M' - open          FMA pipe
      // Ix = max(Ix_left - ext, Mo_left, 0)   (0 at k = 0)  ALU
      // D  = max(M', Ix, Iy, 0)                             ALU
      // Iy(next row) = max(Iy - ext, Mo, 0)                 ALU
      uint32_t X = 0, mo_left = 0;
      uint32_t mp = __vadd2(diag, s[w * TPT]);
#pragma unroll
      for (int k = 0; k < TPT; ++k) {
        const uint32_t mo = __vadd2(mp, nopen2);
        const uint32_t mp_next = (k + 1 < TPT) ? __vadd2(SA[w][k], s[w * TPT + k + 1]) : 0u;
        if (k > 0) X = __viaddmax_s16x2_relu(X, next2, mo_left);
        const uint32_t y = Y[w][k];
        const uint32_t D = (k > 0) ? __vimax3_s16x2_relu(mp, X, y) : __vimax_s16x2_relu(mp, y);
        Y[w][k] = __viaddmax_s16x2_relu(y, next2, mo);
        SA[w][k] = D;
        mo_left = mo;
        mp = mp_next;
        if (((w * TPT + k) & 1) == 0) pend = D;
        else bestA = __vimax3_s16x2(bestA, pend, D);
      }
    }
    if ((L::NWD & 1) != 0) bestA = __vimax_s16x2_relu(bestA, pend);
  };

  // ---- target bytes: R rows at a time from R/4 + 1 aligned 32-bit words.
  // A word is loaded only when it holds a byte of the window being read, so
  // no load leaves the windows' own 4-byte words.
  constexpr int R = rows_per_fetch<MODE, TPT, W>();
  // ---- target bytes and residue classes of the next R rows.  Only bytes
  // inside the window are read; rows past its end are padding rows (class
  // kClsPad).  Where a group has at least R lanes (SPREAD), the lanes share
  // the work: lane gl reads the byte of row gl and turns it into a class,
  // and each row's class is broadcast from its lane with one shuffle (LSU
  // pipe), which keeps the per-byte work off the busy ALU pipe.  Narrower
  // groups read R/4 + 1 aligned 32-bit words per lane, a word only when it
  // holds a byte of the window, and pack four classes per register.
  constexpr bool SPREAD = G >= R;
  constexpr int NB = SPREAD ? 1 : R / 4 + 1;   // bytes (SPREAD) or words per lane
  constexpr uint32_t kNoByte = 0x100u;         // SPREAD: the row is past the end
  constexpr uint32_t kPadWord = kClsPad * 0x01010101u;
  const uintptr_t au = reinterpret_cast<uintptr_t>(a.ascii);
  const uint32_t* abase = reinterpret_cast<const uint32_t*>(au & ~(uintptr_t)3);
  const uint32_t aoff = (uint32_t)(au & 3);
  struct Bytes { uint32_t w[NB]; };
  auto fetch = [&](uint32_t p, uint32_t e) -> Bytes {   // needs p < e
    Bytes q;
    if constexpr (SPREAD) {
      q.w[0] = (gl < R && p + (uint32_t)gl < e) ? (uint32_t)__ldg(a.ascii + p + gl) : kNoByte;
    } else {
      const uint32_t wi = (p + aoff) >> 2;
      q.w[0] = __ldg(abase + wi);
#pragma unroll
      for (int k = 1; k < NB; ++k)
        q.w[k] = ((wi + k) << 2) < e + aoff ? __ldg(abase + wi + k) : 0u;
    }
    return q;
  };
  // In the fused kernel the affine rows may differ from the linear ones in
  // the first row of a target, which is a padding row when the affine
  // windows start one byte later (a padding row from the initial state
  // leaves the state at 0, so this is exactly the later start).
  const bool aff_skip_row = MODE == kBoth && a.skip2 == 1;
  constexpr int NC = SPREAD ? 1 : R / 4;
  uint32_t cw[NC];                    // SPREAD: class of row gl; else 4 per word
  bool pad0 = false;                  // fused kernel: affine row 0 is padding
#pragma unroll
  for (int h = 0; h < NC; ++h) cw[h] = SPREAD ? (uint32_t)kClsPad : kPadWord;
  auto classes = [&](const Bytes& q, uint32_t p, uint32_t e, bool first) {
    if constexpr (SPREAD) {
      cw[0] = q.w[0] < 256u ? (uint32_t)lut[q.w[0]] : (uint32_t)kClsPad;
    } else {
      const uint32_t sh = ((p + aoff) & 3u) * 8u;
#pragma unroll
      for (int h = 0; h < NC; ++h) {
        const uint32_t raw = __funnelshift_r(q.w[h], q.w[h + 1], sh);
        uint32_t word = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const uint32_t cl = p + (4 * h + b) < e ? lut[(raw >> (8 * b)) & 0xffu] : kClsPad;
          word |= cl << (8 * b);
        }
        cw[h] = word;
      }
    }
    if constexpr (MODE == kBoth) pad0 = first && aff_skip_row;
  };
  auto class_of_row = [&](int r) -> int {
    if constexpr (SPREAD) return __shfl_sync(0xffffffffu, (int)cw[0], leader + r);
    else return (int)((cw[r / 4] >> (8 * (r % 4))) & 0xffu);
  };

  // ---- target order (group-uniform).  The group leader takes CH targets
  // at a time from the launch-wide counter; the grab for the chunk after
  // the current one is issued when the current one is taken, and its value
  // is broadcast to the group only when that chunk is reached.  The host
  // sizes CH so that every group gets several chunks.
  // The host splits launches so that n < 2^30: target indices and the
  // counter (which overshoots n by at most two grabs per group) fit 32 bits.
  const int CH = a.chunk;
  const int n = (int)a.n;
  unsigned pre_raw = 0;   // leader only: start of the prefetched chunk
  auto issue_grab = [&]() {
    if (gl == 0) pre_raw = atomicAdd(a.ticket, (unsigned)CH);
  };
  int c_hi;               // end of the chunk the sequence is in
  auto take_chunk = [&]() -> int {
    const int c = (int)__shfl_sync(gmask, pre_raw, leader);
    c_hi = c < n - CH ? c + CH : n;
    if (c < n) issue_grab();
    return c;
  };
  auto successor = [&](int x) -> int {   // next target after x (>= n: none)
    return x + 1 < c_hi ? x + 1 : take_chunk();
  };

  Win cur, nxt;
  int t, tn = 0;
  bool active = false, nxt_ok = false;
  auto start_at = [&](int tt) {   // first target with rows at or after tt
    t = tt;
    while (t < n) {
      cur = window_of(a, t);
      if (cur.rows) break;
      if (gl == 0) {
        if (writeA) a.out[t] = cur.res;
        if constexpr (MODE == kBoth) a.out2[t] = cur.res;
        if constexpr (PAIR) if (writeB) outB[t] = cur.res;
      }
      t = successor(t);
    }
    active = t < n;
    nxt_ok = false;
    if (active) {
      tn = successor(t);
      if (tn < n) { nxt = window_of(a, tn); nxt_ok = true; }
    }
  };
  auto finish = [&](uint32_t best) -> int {   // group maximum of a running max
    int v = max((int)(int16_t)(best & 0xffffu), (int)(int16_t)(best >> 16));
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(gmask, v, o));
    return v;
  };
  auto finish_halves = [&](uint32_t best) -> uint32_t {   // per half (query-pair mode)
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) best = __vmaxs2(best, __shfl_xor_sync(gmask, best, o));
    return best;
  };
  issue_grab();
  start_at(take_chunk());
  if (active) classes(fetch(cur.pos, cur.end), cur.pos, cur.end, true);

  while (__any_sync(0xffffffffu, active)) {
    // prefetch the bytes of the next R rows of this group
    Bytes pf;
#pragma unroll
    for (int k = 0; k < NB; ++k) pf.w[k] = SPREAD ? kNoByte : 0u;
    bool pf_nxt = false;
    if (active) {
      if (cur.pos + R < cur.end) pf = fetch(cur.pos + R, cur.end);
      else if (nxt_ok && nxt.rows) { pf = fetch(nxt.pos, nxt.end); pf_nxt = true; }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int cl = class_of_row(r);
      if constexpr (DO_LIN) row_lin(cl);
      if constexpr (MODE == kAff || MODE == kPair) row_aff(cl);
      if constexpr (MODE == kBoth) row_aff(r == 0 && pad0 ? kClsPad : cl);
    }
    if (active) {
      cur.pos += R;
      if (cur.pos >= cur.end) {
        // target finished (rows past its end were padding rows)
        const int vl = DO_LIN ? finish(bestL) : 0;
        const int va = (DO_AFF && !PAIR) ? finish(bestA) : 0;
        const uint32_t vp = PAIR ? finish_halves(bestA) : 0u;
        if (gl == 0) {
          if constexpr (MODE == kLin) a.out[t] = vl;
          if constexpr (MODE == kAff) a.out[t] = va;
          if constexpr (MODE == kBoth) { a.out[t] = vl; a.out2[t] = va; }
          if constexpr (PAIR) {
            if (writeA) a.out[t] = (int)(int16_t)(vp & 0xffffu);
            if (writeB) outB[t] = (int)(int16_t)(vp >> 16);
          }
        }
        reset();
        if (pf_nxt) {
          t = tn;
          cur = nxt;
          tn = successor(t);
          nxt_ok = tn < n;
          if (nxt_ok) nxt = window_of(a, tn);
          classes(pf, cur.pos, cur.end, true);
        } else {
          start_at(tn);
          if (active) {
            classes(fetch(cur.pos, cur.end), cur.pos, cur.end, true);
          } else {
#pragma unroll
            for (int h = 0; h < NC; ++h) cw[h] = SPREAD ? (uint32_t)kClsPad : kPadWord;
            pad0 = false;
          }
        }
      } else {
        classes(pf, cur.pos, cur.end, false);
      }
    }
  }
}

// ------------------------------------------------------------ registry
using KernelFn = void (*)(SwArgs, const QueryTable);

struct KernelInfo {
  KernelFn fn = nullptr;
  size_t smem = 0;
  int threads = 0;
  int groups_per_block = 0;
  int words = 0;
};

template <int TPT, int MODE, bool WIDE, bool DEF>
KernelInfo make_info() {
  constexpr int W = words_for<TPT, WIDE, MODE>();
  KernelInfo k;
  k.fn = sw_stream_kernel<TPT, W, MODE, DEF>;
  using L = Layout<TPT, W, vector_major<TPT, W, MODE>(), MODE == kPair>;
  k.smem = L::smem + (MODE == kBoth ? L::smem - 256 : 0);
  k.threads = Shape<TPT, W, MODE>::threads;
  k.groups_per_block = (k.threads / 32) * L::GPW;
  k.words = W;
  return k;
}

// tables[gaps][variant][mode][TPT - 1]: gaps 0 = gap parameters read from
// the arguments, 1 = the DEF twin (kDefGap, kDefOpen, kDefExt); variant 0 =
// narrow, 1 = wide; mode kLin, kAff, kBoth or kPair.  The fused kernel
// exists up to kMaxFusedTpt;
// wider queries run the two kernels one after the other (fn == nullptr
// here).  Measured on B200 (300k-1M segments), the fused pass beat the two
// kernels by 4-17% up to width 16 and by 5% at 20 (8 rows per fetch),
// broke even at 27 and lost 13% at 41-48: its three states need ~200-255
// registers there, which leaves 8 warps per SM.  With msa()'s gaps built in
// (1M segments): +7% at 22, +6% at 23, -2% to +2% at 25-32.
constexpr int kMaxFusedTpt = 23;
struct Tables {
  KernelInfo k[2][2][kModes][64];
};

// Instantiations whose DEF twin spills under the register cap (ptxas, 4-8
// bytes) where the runtime-gap kernel does not: their DEF slot holds the
// runtime-gap kernel.
template <int T, int MODE, bool WIDE>
constexpr bool def_twin() {
  return !(MODE == kLin && ((T == 15 && !WIDE) || (T == 23 && WIDE))) &&
         !(MODE == kAff && T == 2 && !WIDE);
}

template <int T, int MODE, bool WIDE, bool DEF>
KernelInfo make_slot() {
  return make_info<T, MODE, WIDE, DEF && def_twin<T, MODE, WIDE>()>();
}

template <int T, bool WIDE, bool DEF>
void fill_one(Tables& t) {
  KernelInfo(&row)[kModes][64] = t.k[DEF][WIDE];
  row[kLin][T - 1] = make_slot<T, kLin, WIDE, DEF>();
  row[kAff][T - 1] = make_slot<T, kAff, WIDE, DEF>();
  if constexpr (T <= kMaxFusedTpt) row[kBoth][T - 1] = make_slot<T, kBoth, WIDE, DEF>();
  row[kPair][T - 1] = make_slot<T, kPair, WIDE, DEF>();
}

template <int LO, bool DEF, int... I>
void fill_range(Tables& t, std::integer_sequence<int, I...>) {
  (fill_one<LO + I, false, DEF>(t), ...);
  (fill_one<LO + I, true, DEF>(t), ...);
}

// Defined in the instantiation units sw_inst_*.cu (runtime gaps) and
// sw_inst_*_def.cu (the DEF twins).
void register_1_16(Tables& t);
void register_17_32(Tables& t);
void register_33_48(Tables& t);
void register_49_64(Tables& t);
void register_1_16_def(Tables& t);
void register_17_32_def(Tables& t);
void register_33_48_def(Tables& t);
void register_49_64_def(Tables& t);

}  // namespace sw
}  // namespace sseqs
