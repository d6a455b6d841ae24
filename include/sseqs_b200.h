/*
 * sseqs_b200.h -- C ABI of libsseqs_b200.so, the B200 (sm_100a) kernels of
 * the sseqs database-search path.
 *
 * Conventions for every entry point:
 *   - all pointers are device pointers unless a comment says "host";
 *   - all work is enqueued on `stream` (0 = legacy default stream); nothing
 *     synchronises unless a comment says so;
 *   - the return value is a status (SSEQS_OK == 0); argument errors are
 *     detected on the host before anything is enqueued;
 *   - no entry point allocates device memory: scratch space is passed in as
 *     `workspace` (size queried with the matching *_workspace_bytes call).
 *
 * Each declaration cites the reference interface it replaces
 * (AlexanderMath/sseqs 0.0.8, file:line).
 */
#ifndef SSEQS_B200_H
#define SSEQS_B200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SSEQS_OK = 0,
  SSEQS_ERR_ARG = 1,          /* invalid argument (null pointer, bad size)   */
  SSEQS_ERR_UNSUPPORTED = 2,  /* valid input outside the supported range     */
  SSEQS_ERR_CUDA = 3,         /* a CUDA runtime call or launch failed        */
  SSEQS_ERR_WORKSPACE = 4,    /* workspace missing or too small              */
  SSEQS_ERR_CAPACITY = 5      /* input larger than a fixed-capacity entry
                                 point can hold (sseqs_topk_static)          */
};

/* Human-readable text for a status code (host, static storage). */
const char* sseqs_status_string(int status);
/* ABI version of this library. */
int sseqs_version(void);
/* Longest query the score kernels accept (2048). */
int sseqs_max_query_len(void);

/* ------------------------------------------------------------------ xbit */
/* 5-bit symbol stream: 8 symbols per 5 bytes, first symbol in the high bits
 * of a big-endian 40-bit window, symbol s <-> byte s+64 ('@' = 0 separates
 * sequences).  Replaces decompress_launcher (sseqs/xbit.cu:65-71, kernel
 * :8-34; torch wrapper sseqs/xbit_bind.cpp:23-28): out[0..n_syms) decodes
 * the stream that starts at packed[lo_bytes]. */
int sseqs_xbit_decompress(const uint8_t* packed, uint8_t* out, int64_t n_syms,
                          int64_t lo_bytes, cudaStream_t stream);
/* Replaces compress_launcher (sseqs/xbit.cu:73-78, kernel :36-62; wrapper
 * sseqs/xbit_bind.cpp:11-18): out holds (5*n_syms+7)/8 bytes; a partial last
 * group packs missing symbols as 0. */
int sseqs_xbit_compress(const uint8_t* in, uint8_t* out, int64_t n_syms,
                        cudaStream_t stream);

/* ------------------------------------------------------ score-only SW
 * Local alignment score of a query (class indices 0..19 in the order
 * ARNDCQEGHILKMFPSTWYV, 1 <= query_len <= 2048) against windows of an ASCII
 * buffer, with BLOSUM62 (non-standard target bytes score -4) and the
 * reference's stripe rule: the horizontal dependency is cut at every query
 * column j with j % ceil(query_len/32) == 0.
 * Target t uses g = good_idx[t] and the window
 *     start = starts[g-1] + 1 (starts[-1] := -1), length = starts[g]-starts[g-1]-1
 * with result -1 when length == 0 or length < -1, and 0 when length == -1
 * (sseqs/sw.cu:66-77, :194-204).  `ascii` must be readable through the end
 * of every 16-byte aligned chunk that holds a byte of some window.
 * out[t] is int32.  query_len > 2048 -> SSEQS_ERR_UNSUPPORTED. */

/* Linear gap (added per gap column; the reference's msa() passes -1).
 * Replaces launch_sw_cuda_blosum62 (sseqs/sw.cu:336-370, kernel :55-179;
 * wrapper sseqs/sw_bind.cpp:32-73). */
int sseqs_sw_linear(const uint8_t* query_idx, int query_len,
                    const int32_t* good_idx, const uint8_t* ascii,
                    const int32_t* starts, int64_t n_targets, int32_t* out,
                    int gap, cudaStream_t stream);

/* Affine gap M/Ix/Iy, gaps open from M only and the first gap column costs
 * gap_open.  Replaces launch_sw_cuda_affine (sseqs/sw.cu:372-425, kernel
 * :182-325; wrapper sseqs/sw_bind.cpp:78-108). */
int sseqs_sw_affine(const uint8_t* query_idx, int query_len,
                    const int32_t* good_idx, const uint8_t* ascii,
                    const int32_t* starts, int64_t n_targets, int32_t* out,
                    int gap_open, int gap_extend, cudaStream_t stream);

/* Both scores above for a database batch held in HBM, in one call shape:
 * target t is segment g = good_idx ? good_idx[t] : g0 + t of the batch whose
 * '@' positions are `delim` (segment g = bytes between delim[g-1] and
 * delim[g]); the first `skip` bytes of each segment are not scored.
 * skip = 0 with delim gives the linear call of sseqs/msa.py:313-319;
 * skip = 1 gives the affine call of sseqs/msa.py:327-332 (which passes
 * delim+1 and so also scores the closing '@' row -- a row that can never
 * raise a local score, so it is not computed). */
int sseqs_sw_scan(int affine, const uint8_t* query_idx, int query_len,
                  const int32_t* good_idx, int32_t g0, int64_t n_targets,
                  const uint8_t* ascii, const int32_t* delim, int skip,
                  int32_t* out, int gap_a, int gap_b, cudaStream_t stream);

/* Both scores of sseqs_sw_scan in one pass: out_linear[t] is the linear
 * score (gap, windows as sseqs_sw_scan with skip 0) and out_affine[t] the
 * affine score (gap_open, gap_extend, windows starting affine_skip (0 or 1)
 * bytes later) of every target -- identical to the two separate calls
 * (the exact search of sseqs/msa.py:313-332 with top_sw = 1 makes both),
 * including query_len 0, where every result of both is -1.
 * Gap parameters must lie in the int16 domain, else SSEQS_ERR_UNSUPPORTED
 * (make the two calls instead).  Queries of up to 736 residues run one
 * fused kernel; longer ones run the two score kernels in turn.
 * Like every single-query scan, it takes its target counter from a ring of
 * 1024 library-owned slots, one per launch: eager calls overlapping on
 * other streams never share one, but a call captured into a CUDA graph
 * keeps its slot for every replay, so a replay must not overlap other
 * single-query scans (the batched call below takes caller-owned counters
 * and has no such limit). */
int sseqs_sw_scan_both(const uint8_t* query_idx, int query_len, const int32_t* good_idx,
                       int32_t g0, int64_t n_targets, const uint8_t* ascii, const int32_t* delim,
                       int affine_skip, int32_t* out_linear, int32_t* out_affine, int gap,
                       int gap_open, int gap_extend, cudaStream_t stream);

/* sseqs_sw_scan for several queries of one stripe width against one batch,
 * in one launch per 128 queries (the batched path; the reference runs one
 * query at a time, sseqs/msa.py:235).  Query i has query_lens[i] (device
 * int32) residue classes at queries + i * query_stride (device), scores the
 * targets of sseqs_sw_scan -- with good_idx + i * idx_stride as its list
 * when good_idx is given (idx_stride 0: one list for all, else >=
 * n_targets) -- and writes its scores to out + i * out_stride (out_stride
 * >= n_targets).  Every length
 * must satisfy ceil(len/32) == tpt and len <= query_stride; a query that does
 * not is not scored and its row is filled with INT32_MIN.  tickets: device
 * scratch of n_queries uint32 (target counters, zeroed by the call on
 * `stream`).  Gap parameters must lie in the int16 domain (linear -16384 <=
 * gap <= 0; affine 0 <= open, extend <= 16384), else SSEQS_ERR_UNSUPPORTED.
 * Every query's scores are identical to its own sseqs_sw_scan call.  The
 * lengths are read on the device, so a captured CUDA graph can be replayed
 * with other queries of the same width.
 * Affine queries that share their targets (good_idx null or idx_stride 0)
 * are scored two per launch row: query 2y in the low and query 2y + 1 in the
 * high half of every int16x2 word, one target fetch and profile-row load for
 * both, at the widths sseqs_sw_set_query_pairing selects; scores are the
 * same. */
int sseqs_sw_scan_queries(int affine, int n_queries, int tpt, const uint8_t* queries,
                          int64_t query_stride, const int32_t* query_lens,
                          const int32_t* good_idx, int64_t idx_stride, int32_t g0,
                          int64_t n_targets,
                          const uint8_t* ascii, const int32_t* delim, int skip,
                          int32_t* out, int64_t out_stride, int gap_a, int gap_b,
                          uint32_t* tickets, cudaStream_t stream);

/* ------------------------------------------------------------ selection */
/* Positions (int32, increasing) of every '@' (64) byte of a decoded batch:
 * replaces `delim_pos = arange[ascii == 64]` (sseqs/msa.py:227).  Writes at
 * most max_out positions and the total count to *count (device int64).
 * n must be < 2^31 (positions are batch-local int32 as in the reference). */
size_t sseqs_find_delims_workspace_bytes(int64_t n);
int sseqs_find_delims(const uint8_t* ascii, int64_t n, int32_t* out_pos, int64_t max_out,
                      int64_t* count, void* workspace, size_t ws_bytes, cudaStream_t stream);

/* Segment table of one decoded batch (sseqs/msa.py:237-267): with the
 * '@' positions `delim` (*n_delims of them, device), segment k ends at
 * delim[k] (plus a trailing segment when the batch does not end in '@');
 * the non-empty ones are listed in order: seg_index[f] = k, lengths[f],
 * offsets[f] = sum over earlier non-empty segments of (length+1) -- the
 * reference's `_offsets` -- with their count in *n_segments and the largest
 * length in *maxlen (all device).  Every output holds max_segments slots
 * (>= number of '@' + 1). */
size_t sseqs_segment_table_workspace_bytes(int64_t max_segments);
int sseqs_segment_table(const uint8_t* ascii, int64_t n, const int32_t* delim,
                        const int64_t* n_delims, int64_t max_segments, int32_t* seg_index,
                        int32_t* lengths, int64_t* offsets, int64_t* n_segments, int32_t* maxlen,
                        void* workspace, size_t ws_bytes, cudaStream_t stream);

/* Indices (int32, increasing) of the k largest of n keys; key_type 0 =
 * int32, 1 = IEEE half.  Ties at the k-th value are taken lowest index
 * first.  Replaces torch.topk + torch.sort of the candidate lists
 * (sseqs/msa.py:297, 307, 324, 335), whose tie order is unspecified.
 * Requires 0 <= k <= n < 2^31. */
size_t sseqs_topk_workspace_bytes(int64_t n);
int sseqs_topk(const void* keys, int key_type, int64_t n, int64_t k, int32_t* out_idx,
               void* workspace, size_t ws_bytes, cudaStream_t stream);

/* Same selection as sseqs_topk, for callers that must not allocate device
 * memory: code whose GPU memory is owned by another allocator (a framework's
 * caching pool, a server's fixed budget) and may not take memory behind its
 * back, or a latency-critical caller that cannot afford the stalls that
 * cudaMalloc / cudaFree can cause.  The caller passes keys and out_idx only;
 * the scratch is a fixed array inside this library (about 66 KB per GPU that
 * loads the library, held until the process exits), so n is limited to
 * SSEQS_TOPK_STATIC_MAX_N keys -- larger n returns SSEQS_ERR_CAPACITY.  The
 * first call on a device looks up that array's device address (with the
 * device current); make that first call before any stream capture.  All
 * calls share the one array: calls that overlap on the GPU (other streams,
 * other host threads) race and must be serialised by the caller.  Nothing
 * is allocated, neither here nor in the kernels.
 * This entry point has no counterpart in the reference. */
#define SSEQS_TOPK_STATIC_MAX_N (1 << 24)
int sseqs_topk_static(const void* keys, int key_type, int64_t n, int64_t k, int32_t* out_idx,
                      cudaStream_t stream);

/* Packs segments of several resident buffers into one: segment i, the
 * len[i] bytes at byte src[i] of the buffer whose device address is
 * bases[part[i]], is copied to out + dst[i] and followed by one '@' (the
 * caller chooses dst so that segments do not overlap, e.g. the exclusive
 * running sum of len + 1).  With delim[i] = dst[i] + len[i] the packed buffer
 * is a database batch of its own whose segment i is segment i of the list,
 * so candidates from many batches can be scored in one launch.  No
 * reference counterpart (the reference scores one batch at a time,
 * sseqs/msa.py:235). */
int sseqs_pack_segments(const uint64_t* bases, const int32_t* part, const int64_t* src,
                        const int32_t* len, const int64_t* dst, int64_t n, uint8_t* out,
                        cudaStream_t stream);

/* Hit strings of selected segments: row r of out (width bytes) receives
 * ascii[offsets[g] .. offsets[g] + min(width, lengths[g])), g = idx[r], the
 * rest of the row zero, and out_len[r] the copied length.  Replaces the
 * gather of sseqs/msa.py:349-370 (width 500 there, sseqs/msa.py:183). */
int sseqs_gather_windows(const uint8_t* ascii, const int64_t* offsets, const int32_t* lengths,
                         const int32_t* idx, int64_t n, int width, uint8_t* out,
                         int32_t* out_len, cudaStream_t stream);

/* ------------------------------------------------------------ traceback */
/* Affine local alignment with traceback of one query (raw bytes) against B
 * targets (bytes at tbytes + toff[b], tlen[b] <= max_target_len each):
 * replaces the Triton kernels sseqs/sw.py:408-563 (DP) and :569-768
 * (traceback) driven by sseqs/sw.py:27-219.  Textbook Gotoh with gaps
 * opening from H, BLOSUM62 for upper-case standard residues else -5.
 * Outputs: best[b]; info[b*5 + 0..4] = alignment length, query start, query
 * end, target start, target end (0-based, -1 when no alignment); the
 * aligned query/target bytes ('-' for gaps) in the LAST `length` bytes of
 * row b of q_aligned/t_aligned (cap >= query_len + max_target_len bytes per
 * row).  m_full (nullable) receives M(i,j) as int32 in a [B][query_len+1]
 * [tcols] array the caller zero-filled.  A target longer than
 * max_target_len gets best = -1. */
size_t sseqs_backtrack_workspace_bytes(int query_len, int max_target_len, int B);
int sseqs_backtrack_affine(const uint8_t* query, int query_len, const uint8_t* tbytes,
                           const int64_t* toff, const int32_t* tlen, int max_target_len, int B,
                           int gap_open, int gap_extend, int32_t* best, int32_t* info,
                           uint8_t* q_aligned, uint8_t* t_aligned, int cap, int32_t* m_full,
                           int tcols, void* workspace, size_t ws_bytes, cudaStream_t stream);

/* a3m rows of traceback results (host function; every pointer is host
 * memory).  Row k is the alignment q_rows[k][0..lens[k]) / t_rows[k][..)
 * (ASCII bytes, '-' for gaps) with integer score scores[k]; rows are taken
 * in order[0..n_rows) (the caller's descending sort of the scores).  Each
 * kept row is written as ">target_<i> score=<score>.0\n<row>\n" where i is
 * its position in `order` and <row> places the alignment at the first
 * occurrence of its gap-free query fragment in `query`, padded with '-' to
 * the query's length, target residues upper case against a query residue
 * and lower case against a query gap.  Rows with score 0 or no alignment,
 * rows holding '@' and repeats of an earlier row are skipped.  Replaces the
 * row loop of to_a3m (sseqs/to_a3m.py:16-72).  *out_len receives the bytes
 * written to out; SSEQS_ERR_UNSUPPORTED when a fragment does not occur in
 * the query (the reference raises ValueError), SSEQS_ERR_CAPACITY when
 * out_cap is too small. */
int sseqs_a3m_rows(const char* query, int64_t query_len, int64_t n_rows, const int64_t* order,
                   const uint8_t* const* q_rows, const uint8_t* const* t_rows,
                   const int32_t* lens, const int64_t* scores, char* out, int64_t out_cap,
                   int64_t* out_len);

/* ------------------------------------------------------------ prefilter */
/* Gapless rank-k correlation score of every segment (fp16 out[s]):
 * 0.5 * max over even lags of sum_r (a_r (*) b_r), a cyclic convolution of
 * length n (power of two, 64..2048), a_r[i] = lut_a[r][query_pos_reversed[i]],
 * b_r[i] = lut_b[r][pos(t[i])] over the segment's bytes ascii[offsets[s] ..
 * + lengths[s]); lut_a / lut_b are float [k][21] (k <= 20).  Replaces
 * launch_warp_corr (sseqs/filter.cu:161-395 with kernels
 * sseqs/filter.cu:92-159 and sseqs/fft.cu:17-415, wrapper
 * sseqs/filter_bind.cpp:20-64); computed in fp32. */
size_t sseqs_prefilter_workspace_bytes(int n, int k);
int sseqs_prefilter(const uint8_t* ascii, const int64_t* offsets, const int32_t* lengths,
                    int64_t n_segments, const uint8_t* query_pos_reversed, int query_len,
                    const float* lut_a, const float* lut_b, int k, int n, void* out,
                    void* workspace, size_t ws_bytes, cudaStream_t stream);

/* --------------------------------------------------------- diagnostics */
/* Measured int16x2 DPX issue rate of this GPU: runs a fixed kernel of
 * independent __viaddmax_s16x2_relu/__vimax3_s16x2 chains and writes
 * (host) the rate in lane-instructions per second.  `sink` is one device
 * word the kernel may write so that its work is not optimised away.
 * Synchronises on `stream`.  No reference counterpart (measurement aid). */
int sseqs_dpx_peak(uint32_t* sink, double* lane_ops_per_s, cudaStream_t stream);
/* int16x2 issue rate over both int pipes: max-type DPX instructions (ALU
 * pipe) interleaved with int16x2 adds (FMA pipe), in lane-instructions per
 * second.  Synchronises.  No reference counterpart (measurement aid). */
int sseqs_int16x2_peak(uint32_t* sink, double* lane_ops_per_s, cudaStream_t stream);
/* Number of kernels this library has enqueued since it was loaded (every
 * launch site counts itself).  No reference counterpart. */
int64_t sseqs_launch_count(void);

/* ----------------------------------------------------------- tuning */
/* The score kernel has two lane layouts for stripe widths tpt =
 * ceil(query_len/32) <= 16: narrow (wide = 0, default) and wide (wide = 1:
 * twice the columns per lane, twice the targets per warp).  Selects the one
 * used for (affine, tpt) -- affine 0 linear, 1 affine, 2 the fused pass, 3
 * the query-pair kernel of sseqs_sw_scan_queries; both give identical
 * scores.  No reference
 * counterpart (the autotuner of the batched path sets it). */
int sseqs_sw_set_variant(int affine, int tpt, int wide);
/* Whether sseqs_sw_scan_queries scores affine queries of stripe width tpt
 * (0: every width) that share their targets two per launch row (on = 1) or
 * one (0, the default until the autotuner of the batched path has timed
 * both); scores are the same either way.  The getter returns the setting,
 * or -1 for a width out of range.  No reference counterpart (the reference
 * scores one query at a time). */
int sseqs_sw_set_query_pairing(int tpt, int on);
int sseqs_sw_get_query_pairing(int tpt);
/* The layout currently selected for (affine, tpt): 0 or 1; -1 if out of
 * range.  No reference counterpart. */
int sseqs_sw_get_variant(int affine, int tpt);
/* int16x2 words per lane of a variant (for reports); -1 if out of range. */
int sseqs_sw_variant_words(int affine, int tpt, int wide);

/* ------------------------------------------------- learned prefilter
 * No reference counterpart: a trained embedding stands in for the FFT
 * prefilter stage (sseqs/msa.py:110-307) as a way to choose candidates for
 * exact SW.  Layout of a set of sequences: row-major bf16 [P x C]
 * activations, each sequence followed by >= 2 zero rows and preceded by 2
 * (row0 of the first sequence >= 2), buffers with 2 addressable zero rows
 * before row 0 and after row P-1.  Classes: 0..19 ARNDCQEGHILKMFPSTWYV,
 * 20 other residues, 255 padding.  bf16 data are __nv_bfloat16. */

/* C = op(A) . op(B)^T over K (K % 32 == 0): A is [M x K] (a_t = 0, row
 * stride lda) or stored [K x M] (a_t = 1); B is [N x K] (b_t = 0) or
 * stored [K x N] (b_t = 1); supported (a_t, b_t): (0, 0) with epilogues
 * 0-3, (1, 1) with epilogues 0 and 4.  Epilogue 0: C fp32; 1: C bf16;
 * 2: C2 = acc + bias (bf16 pre-activation), C = GELU(C2) (bf16, tanh form);
 * 3: C = acc * GELU'(aux) (bf16, aux bf16 with C's stride); 4: C (fp32,
 * zeroed by the caller) += acc with K split over CTAs (for small M x N and
 * long K, as in weight gradients); 5: as 2 with res (bf16, C's stride) added
 * to C (a residual connection); 6: C2 = acc + res, C = C2 * GELU'(aux) (the
 * gradient through a residual connection).  Epilogues 5 and 6 need
 * (a_t, b_t) = (0, 0).  row_mask
 * (nullable, uint8 per row of C): rows with 0 are written as 0 (epilogues
 * 1-3).  A, B 16-byte aligned, lda, ldb multiples of 8; a_t needs M % 8 ==
 * 0, b_t N % 8 == 0.  Tensor cores (mma.sync bf16, fp32 accumulation). */
int sseqs_gemm_bf16(int a_t, int b_t, int epilogue, int64_t M, int64_t N, int64_t K,
                    const void* A, int64_t lda, const void* B, int64_t ldb, void* C,
                    int64_t ldc, void* C2, const float* bias, const void* aux,
                    const uint8_t* row_mask, const void* res, cudaStream_t stream);

/* sseqs_gemm_bf16 runs on the 5th-generation tensor cores (tcgen05.mma,
 * fp32 accumulators in tensor memory) when a_t = b_t = 0, N = 256, K is a
 * multiple of 64, ldc a multiple of 8, C/C2/aux/res 16-byte aligned and the
 * epilogue is 1, 2, 3, 5 or 6; otherwise on mma.sync.  set_tensor_path(0)
 * forces mma.sync (1 restores the default).  gemm_error reads and clears the
 * flag a tcgen05 launch sets when one of its bounded waits ran out
 * (synchronous).  A set flag means the tensor-core unit did not answer in
 * time: the launch's output is invalid, and since its last operations were
 * only waited for with a bound, the caller should treat the device state as
 * suspect (stop issuing work and reset the context), not only that output. */
int sseqs_gemm_set_tensor_path(int tcgen05);
int sseqs_gemm_error(int* out);

/* cls[row0[s] + i] = class of ascii[off[s] + i] for i < len[s] (other rows
 * untouched). */
int sseqs_embed_layout(const uint8_t* ascii, const int64_t* off, const int32_t* len,
                       const int64_t* row0, int n_seqs, uint8_t* cls, cudaStream_t stream);
/* The first convolution of the embedder from a table: Z[p] = bf16(bias +
 * sum_{t<5} T[t][cls[p-2+t]]) (fp32 T [5][21][D]: T[t][k] = E[k] . W1[:, t, :]^T;
 * rows outside 0..P-1 and padding classes add nothing), Y[p] = bf16(GELU(Z[p]));
 * rows with row_mask 0 are 0 in both; Z nullable.  Y, Z bf16 [P x D] with row
 * stride D, D % 8 == 0, D <= 512.  No reference counterpart. */
int sseqs_embed_conv1_table(const uint8_t* cls, int64_t P, const float* T, const float* bias,
                            const uint8_t* row_mask, int D, void* Y, void* Z,
                            cudaStream_t stream);
/* X[p][c] = E[cls[p]][c] (bf16, E [21][D]); 0 for padding rows. */
int sseqs_embed_lookup(const uint8_t* cls, int64_t P, const void* E, int D, void* X,
                       cudaStream_t stream);
/* dE[cls[p]][c] += dX[p][c] (fp32 dE, bf16 dX). */
int sseqs_embed_grad(const uint8_t* cls, int64_t P, const void* dX, int D, float* dE,
                     cudaStream_t stream);
/* Per sequence s: pooled = mean of rows start[s] .. + len[s] of Y [P x D]
 * (bf16), emb = pooled / |pooled|, inv_norm = 1 / |pooled| (fp32). */
int sseqs_pool_normalize(const void* Y, int D, const int64_t* start, const int32_t* len,
                         int n_seqs, float* pooled, float* emb, float* inv_norm,
                         cudaStream_t stream);
/* For B pairs with weights w (weight nullable: 1/B each): pred =
 * <emb[ia], emb[ib]>, *loss += w (pred - y)^2, and (dE non-null) dE[ia] +=
 * 2 w (pred - y) emb[ib], dE[ib] likewise; pred (nullable) receives the dot
 * products. */
int sseqs_pair_loss(const float* emb, int D, const int32_t* ia, const int32_t* ib,
                    const float* y, const float* weight, int64_t B, float* dE, float* loss,
                    float* pred, cudaStream_t stream);
/* Gradient of pool_normalize back to the last layer: for the rows of every
 * sequence (other rows untouched) dY = (dE - emb <emb, dE>) * inv_norm /
 * len, stored in G when G is non-null, and dZ = dY * GELU'(Z). */
int sseqs_pool_backward(const float* emb, const float* dE, const float* inv_norm,
                        const int64_t* start, const int32_t* len, int n_seqs, int D,
                        const void* Z, void* dZ, void* G, cudaStream_t stream);
/* db[c] += sum over the P rows of dZ[p][c]. */
int sseqs_bias_grad(const void* dZ, int64_t P, int D, float* db, cudaStream_t stream);
/* Adam step of a conv weight W[Cout][5][Cin] (fp32 w, m, v) from dWT
 * [5*Cin][Cout] (the weight-grad GEMM's output); writes bf16 Wb[co][t][ci]
 * and Wf[ci][4-t][co]. */
int sseqs_adam_conv(float* w, float* m, float* v, const float* dWT, int Cout, int Cin, float lr,
                    float b1, float b2, float eps, int step, void* Wb, void* Wf,
                    cudaStream_t stream);
/* Adam step of n flat parameters; wb (nullable) receives a bf16 copy. */
int sseqs_adam_flat(float* w, float* m, float* v, const float* g, int64_t n, float lr, float b1,
                    float b2, float eps, int step, void* wb, cudaStream_t stream);
/* out[i] = e4m3 code of scale * x[i] (saturating). */
int sseqs_quantize_e4m3(const float* x, int64_t n, float scale, uint8_t* out,
                        cudaStream_t stream);
/* Candidate selection by FP8 GEMM (e4m3, fp32 accumulation): for every
 * query q (codes Q [nq][256]) and database row r (codes DB [n][256]) with
 * <Q[q], DB[r]> >= tau[q], appends r (and the dot product) to q's list:
 * slot = count[q]++ (count zeroed by the caller), kept when slot < cap, at
 * cand[q*cap + slot] / cand_score[q*cap + slot]; list order is not fixed.
 * Q, DB 16-byte aligned.  Runs on tcgen05.mma kind::f8f6f4 (database rows
 * as M = 128, queries as N = nq rounded up to 16, at most 256 per tile, TMA
 * loads) unless sseqs_gemm_set_tensor_path(0) selected mma.sync; a bounded
 * wait that ran out sets the flag sseqs_gemm_error reads. */
int sseqs_score_select(const uint8_t* Q, int nq, const uint8_t* DB, int64_t n, const float* tau,
                       int32_t* count, int64_t* cand, float* cand_score, int cap,
                       cudaStream_t stream);
/* Dense dot products out[q][r] = <Q[q], DB[r]> (fp32, [nq][n]). */
int sseqs_score_dense(const uint8_t* Q, int nq, const uint8_t* DB, int64_t n, float* out,
                      cudaStream_t stream);
/* out[r] = k-th largest of row r of x [rows][n] (n <= 8192). */
int sseqs_kth_largest_rows(const float* x, int rows, int n, int k, float* out,
                           cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* SSEQS_B200_H */
