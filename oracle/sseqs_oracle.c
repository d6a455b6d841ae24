/*
 * sseqs_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C CPU restatement of the reference (AlexanderMath/sseqs 0.0.8)
 * algorithms on the database-search path.  It is the checker for the CUDA
 * product in sseqs_b200/: only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it.  The product never links or calls it.
 *
 * Every function cites the reference file:line it restates:
 *   - xbit 5-bit codec ............ sseqs/xbit.cu:8-62
 *   - linear score-only SW ........ sseqs/sw.cu:55-179  (launcher :336-370)
 *   - affine score-only SW ........ sseqs/sw.cu:182-325 (launcher :372-425)
 *   - textbook affine DP+traceback  sseqs/sw.py:27-219, :408-563, :569-768
 *
 * Deliberate, documented deviations (all on inputs where the reference reads
 * out of bounds, i.e. has no defined result):
 *   - target index g == 0: the reference reads starts[-1] (sw.cu:69,197);
 *     here starts[-1] is taken as -1, so window 0 begins at byte 0.
 *   - target bytes >= 128: the reference indexes its table with a signed
 *     char (sw.cu:116-117); here such bytes are "unknown" (score -4).
 *   - xbit n % 8 != 0: the reference reads/writes past the buffers
 *     (xbit.cu:18,44); here the tail is bounds-checked.
 *   - query length 1024 < Lq <= 2048: the reference launches nothing
 *     (sw.cu:357-369); here the same stripe rule is extended
 *     (TPT = ceil(Lq/32)).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* BLOSUM62 in the residue order ARNDCQEGHILKMFPSTWYV (published matrix;
 * the same table the reference embeds at sw.cu:7-29 and msa.py:110). */
static const int8_t B62[20][20] = {
    { 4,-1,-2,-2, 0,-1,-1, 0,-2,-1,-1,-1,-1,-2,-1, 1, 0,-3,-2, 0},
    {-1, 5, 0,-2,-3, 1, 0,-2, 0,-3,-2, 2,-1,-3,-2,-1,-1,-3,-2,-3},
    {-2, 0, 6, 1,-3, 0, 0, 0, 1,-3,-3, 0,-2,-3,-2, 1, 0,-4,-2,-3},
    {-2,-2, 1, 6,-3, 0, 2,-1,-1,-3,-4,-1,-3,-3,-1, 0,-1,-4,-3,-3},
    { 0,-3,-3,-3, 9,-3,-4,-3,-3,-1,-1,-3,-1,-2,-3,-1,-1,-2,-2,-1},
    {-1, 1, 0, 0,-3, 5, 2,-2, 0,-3,-2, 1, 0,-3,-1, 0,-1,-2,-1,-2},
    {-1, 0, 0, 2,-4, 2, 5,-2, 0,-3,-3, 1,-2,-3,-1, 0,-1,-3,-2,-2},
    { 0,-2, 0,-1,-3,-2,-2, 6,-2,-4,-4,-2,-3,-3,-2, 0,-2,-2,-3,-3},
    {-2, 0, 1,-1,-3, 0, 0,-2, 8,-3,-3,-1,-2,-1,-2,-1,-2,-2, 2,-3},
    {-1,-3,-3,-3,-1,-3,-3,-4,-3, 4, 2,-3, 1, 0,-3,-2,-1,-3,-1, 3},
    {-1,-2,-3,-4,-1,-2,-3,-4,-3, 2, 4,-2, 2, 0,-3,-2,-1,-2,-1, 1},
    {-1, 2, 0,-1,-3, 1, 1,-2,-1,-3,-2, 5,-1,-3,-1, 0,-1,-3,-2,-2},
    {-1,-1,-2,-3,-1, 0,-2,-3,-2, 1, 2,-1, 5, 0,-2,-1,-1,-1,-1, 1},
    {-2,-3,-3,-3,-2,-3,-3,-3,-1, 0, 0,-3, 0, 6,-4,-2,-2, 1, 3,-1},
    {-1,-2,-2,-1,-3,-1,-1,-2,-2,-3,-3,-1,-2,-4, 7,-1,-1,-4,-3,-2},
    { 1,-1, 1, 0,-1, 0, 0, 0,-1,-2,-2, 0,-1,-2,-1, 4, 1,-3,-2,-2},
    { 0,-1, 0,-1,-1,-1,-1,-2,-2,-1,-1,-1,-1,-2,-1, 1, 5,-2,-2, 0},
    {-3,-3,-4,-4,-2,-2,-3,-2,-2,-3,-2,-3,-1, 1,-4,-3,-2,11, 2,-3},
    {-2,-2,-2,-3,-2,-1,-2,-3, 2,-1,-1,-2,-1, 3,-3,-2,-2, 2, 7,-1},
    { 0,-3,-3,-3,-1,-2,-2,-3,-3, 3, 1,-2, 1,-1,-2,-2, 0,-3,-1, 4},
};

static const char AA[20] = {'A','R','N','D','C','Q','E','G','H','I',
                            'L','K','M','F','P','S','T','W','Y','V'};

/* ASCII -> residue class 0..19, -1 for anything else (sw.cu:31-53). */
static int aa_class(uint8_t c) {
    for (int k = 0; k < 20; ++k)
        if ((uint8_t)AA[k] == c) return k;
    return -1;
}

int oracle_version(void) { return 1; }

/* ------------------------------------------------------------------ */
/* xbit codec (xbit.cu:8-34 decompress, xbit.cu:36-62 compress)        */
/* ------------------------------------------------------------------ */

/* 5 packed bytes hold 8 symbols, first symbol in the high bits of a
 * 40-bit big-endian window; symbol s decodes to the byte s + 64. */
void oracle_xbit_decompress(const uint8_t* packed, uint8_t* out,
                            int64_t n_syms, int64_t lo_bytes) {
    const uint8_t* in = packed + lo_bytes;
    for (int64_t t = 0; t * 8 < n_syms; ++t) {
        const uint8_t* p = in + t * 5;
        uint64_t w = ((uint64_t)p[0] << 32) | ((uint64_t)p[1] << 24) |
                     ((uint64_t)p[2] << 16) | ((uint64_t)p[3] << 8) |
                     (uint64_t)p[4];
        for (int k = 0; k < 8 && t * 8 + k < n_syms; ++k)
            out[t * 8 + k] = (uint8_t)(((w >> (35 - 5 * k)) & 31u) + 64u);
    }
}

/* Inverse of the above.  Output holds (5*n+7)/8 bytes; a partial final
 * group packs the missing symbols as 0 ('@'). */
void oracle_xbit_compress(const uint8_t* in, uint8_t* out, int64_t n_syms) {
    int64_t out_bytes = (n_syms * 5 + 7) / 8;
    for (int64_t t = 0; t * 8 < n_syms; ++t) {
        uint64_t w = 0;
        for (int k = 0; k < 8; ++k) {
            uint8_t s = (t * 8 + k < n_syms) ? (uint8_t)(in[t * 8 + k] - 64u) : 0;
            w |= (uint64_t)(s & 31u) << (35 - 5 * k);
        }
        for (int b = 0; b < 5; ++b)
            if (t * 5 + b < out_bytes)
                out[t * 5 + b] = (uint8_t)(w >> (32 - 8 * b));
    }
}

/* ------------------------------------------------------------------ */
/* Score-only SW with the reference's stripe rule                      */
/* ------------------------------------------------------------------ */
/*
 * The reference kernel gives each of the 32 lanes of a warp a stripe of
 * TPT = roundup32(Lq)/32 consecutive query columns and advances all lanes
 * row by row (one target residue per row).  At the first column of every
 * stripe the left neighbour H(i, j-1) is taken as 0 (sw.cu:118, :250);
 * the diagonal neighbour crosses stripes through a shuffle (sw.cu:111-113,
 * :241-246).  Row-major, that is a textbook DP whose horizontal dependency
 * is cut at every column j with j % TPT == 0 -- which is what is written
 * below.  Window of target t (sw.cu:69-77, :197-204):
 *     start = starts[g-1] + 1, stop = starts[g] + 1, length = stop-start-1
 *     score -1 if Lq == 0, length == 0 or stop < start.
 */

typedef struct {
    int64_t start;
    int64_t length;   /* may be <= 0 */
    int special;      /* 1 -> result is -1 without computing */
} window_t;

static window_t ref_window(const int32_t* starts, int32_t g) {
    window_t w;
    int64_t prev = (g == 0) ? -1 : (int64_t)starts[g - 1];
    int64_t start = prev + 1;
    int64_t stop = (int64_t)starts[g] + 1;
    w.start = start;
    w.length = stop - start - 1;
    w.special = (w.length == 0 || stop < start);
    return w;
}

/* Linear gap, uint16 cells (sw.cu:55-179). */
static int32_t sw_linear_one(const uint8_t* q, int Lq, const uint8_t* t,
                             int64_t len, int gap, uint16_t* prev,
                             uint16_t* cur) {
    const int TPT = (Lq + 31) / 32;
    int32_t best = 0;
    memset(prev, 0, sizeof(uint16_t) * (size_t)Lq);
    for (int64_t i = 0; i < len; ++i) {
        int c = aa_class(t[i]);
        uint16_t left = 0;
        for (int j = 0; j < Lq; ++j) {
            int s = (c < 0) ? -4 : B62[c][q[j]];
            int diag = (j == 0) ? 0 : prev[j - 1];
            int up = prev[j];
            int lft = (j % TPT == 0) ? 0 : left;
            int h = diag + s;
            if (up + gap > h) h = up + gap;
            if (lft + gap > h) h = lft + gap;
            if (h < 0) h = 0;
            uint16_t h16 = (uint16_t)h;
            cur[j] = h16;
            if (h16 > best) best = h16;
            left = h16;
        }
        memcpy(prev, cur, sizeof(uint16_t) * (size_t)Lq);
    }
    return best;
}

/* Affine gap M/Ix/Iy, int16 cells (sw.cu:182-325).
 *   M  = max(0, max(M,Ix,Iy)(i-1,j-1) + s)
 *   Ix = max(0, M(i,j-1) - open, Ix(i,j-1) - ext)   [left; cut at stripes]
 *   Iy = max(0, M(i-1,j) - open, Iy(i-1,j) - ext)   [up]
 *   score = max over cells of max(M, Ix, Iy)                              */
static int32_t sw_affine_one(const uint8_t* q, int Lq, const uint8_t* t,
                             int64_t len, int gap_open, int gap_extend,
                             int16_t* pM, int16_t* pX, int16_t* pY,
                             int16_t* cM, int16_t* cX, int16_t* cY) {
    const int TPT = (Lq + 31) / 32;
    int32_t best = 0;
    memset(pM, 0, sizeof(int16_t) * (size_t)Lq);
    memset(pX, 0, sizeof(int16_t) * (size_t)Lq);
    memset(pY, 0, sizeof(int16_t) * (size_t)Lq);
    for (int64_t i = 0; i < len; ++i) {
        int c = aa_class(t[i]);
        int16_t lM = 0, lX = 0;
        for (int j = 0; j < Lq; ++j) {
            int s = (c < 0) ? -4 : B62[c][q[j]];
            int dM = 0, dX = 0, dY = 0;
            if (j > 0) { dM = pM[j - 1]; dX = pX[j - 1]; dY = pY[j - 1]; }
            if (j % TPT == 0) { lM = 0; lX = 0; }
            int m = dM + s;
            if (dX + s > m) m = dX + s;
            if (dY + s > m) m = dY + s;
            if (m < 0) m = 0;
            int x = lM - gap_open;
            if (lX - gap_extend > x) x = lX - gap_extend;
            if (x < 0) x = 0;
            int y = pM[j] - gap_open;
            if (pY[j] - gap_extend > y) y = pY[j] - gap_extend;
            if (y < 0) y = 0;
            int16_t m16 = (int16_t)m, x16 = (int16_t)x, y16 = (int16_t)y;
            cM[j] = m16; cX[j] = x16; cY[j] = y16;
            int mx = m16;
            if (x16 > mx) mx = x16;
            if (y16 > mx) mx = y16;
            if (mx > best) best = mx;
            lM = m16; lX = x16;
        }
        memcpy(pM, cM, sizeof(int16_t) * (size_t)Lq);
        memcpy(pX, cX, sizeof(int16_t) * (size_t)Lq);
        memcpy(pY, cY, sizeof(int16_t) * (size_t)Lq);
    }
    return best;
}

typedef struct {
    const uint8_t* q; int Lq;
    const int32_t* good_idx; int64_t n;
    const uint8_t* ascii; const int32_t* starts;
    int32_t* out;
    int affine, p0, p1;
    int64_t lo, hi;
} sw_job_t;

static void* sw_job_run(void* arg) {
    sw_job_t* jb = (sw_job_t*)arg;
    int Lq = jb->Lq;
    int16_t* buf = (int16_t*)malloc(sizeof(int16_t) * 6 * (size_t)(Lq > 0 ? Lq : 1));
    for (int64_t k = jb->lo; k < jb->hi; ++k) {
        window_t w = ref_window(jb->starts, jb->good_idx[k]);
        if (Lq == 0 || Lq > 2048 || w.special) { jb->out[k] = -1; continue; }
        if (w.length < 0) { jb->out[k] = 0; continue; }   /* loop runs 0 rows */
        const uint8_t* t = jb->ascii + w.start;
        if (jb->affine)
            jb->out[k] = sw_affine_one(jb->q, Lq, t, w.length, jb->p0, jb->p1,
                                       buf, buf + Lq, buf + 2 * Lq,
                                       buf + 3 * Lq, buf + 4 * Lq, buf + 5 * Lq);
        else
            jb->out[k] = sw_linear_one(jb->q, Lq, t, w.length, jb->p0,
                                       (uint16_t*)buf, (uint16_t*)(buf + Lq));
    }
    free(buf);
    return NULL;
}

static int sw_run(const uint8_t* q, int Lq, const int32_t* good_idx,
                  int64_t n, const uint8_t* ascii, const int32_t* starts,
                  int32_t* out, int affine, int p0, int p1, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 1024) nthreads = 1024;
    for (int j = 0; j < Lq; ++j)
        if (q[j] >= 20) return 1;   /* query must hold class indices 0..19 */
    sw_job_t jobs[1024];
    pthread_t th[1024];
    int64_t per = (n + nthreads - 1) / nthreads;
    int launched = 0;
    for (int i = 0; i < nthreads; ++i) {
        sw_job_t* jb = &jobs[i];
        jb->q = q; jb->Lq = Lq; jb->good_idx = good_idx; jb->n = n;
        jb->ascii = ascii; jb->starts = starts; jb->out = out;
        jb->affine = affine; jb->p0 = p0; jb->p1 = p1;
        jb->lo = (int64_t)i * per;
        jb->hi = jb->lo + per < n ? jb->lo + per : n;
        if (jb->lo >= jb->hi) break;
        if (nthreads == 1) { sw_job_run(jb); launched = 0; break; }
        pthread_create(&th[i], NULL, sw_job_run, jb);
        launched++;
    }
    for (int i = 0; i < launched; ++i) pthread_join(th[i], NULL);
    return 0;
}

/* Reference-window semantics of sw_cuda_blosum62 (sw_bind.cpp:32-73). */
int oracle_sw_linear(const uint8_t* q_idx, int Lq, const int32_t* good_idx,
                     int64_t n, const uint8_t* ascii, const int32_t* starts,
                     int32_t* out, int gap, int nthreads) {
    return sw_run(q_idx, Lq, good_idx, n, ascii, starts, out, 0, gap, 0, nthreads);
}

/* Reference-window semantics of sw_cuda_affine (sw_bind.cpp:78-108). */
int oracle_sw_affine(const uint8_t* q_idx, int Lq, const int32_t* good_idx,
                     int64_t n, const uint8_t* ascii, const int32_t* starts,
                     int32_t* out, int gap_open, int gap_extend, int nthreads) {
    return sw_run(q_idx, Lq, good_idx, n, ascii, starts, out, 1, gap_open,
                  gap_extend, nthreads);
}

/* ------------------------------------------------------------------ */
/* Textbook affine DP + traceback (sw.py Triton kernels)                */
/* ------------------------------------------------------------------ */
/*
 * DP (sw.py:505-536), i = query position, j = target position, 1-based:
 *   H(i,j)  = max(0, M, Ix, Iy), borders (row/col 0) are 0
 *   M(i,j)  = s(q_i, t_j) + H(i-1,j-1)
 *   Ix(i,j) = max(H(i-1,j) - open, Ix(i-1,j) - ext), Ix(0,j) := -16384
 *   Iy(i,j) = max(H(i,j-1) - open, Iy(i,j-1) - ext), Iy(i,0) := -16384
 *   s = BLOSUM62 for two standard upper-case residues, else -5
 *   (sw.py:254-260, :498-503).  Cells are int16 (sw.py:62-64).
 * Traceback (sw.py:612-768): end cell = first (i,j) in query-major order
 * with H == best; then repeat: stop if H == 0 or at a border; H == M ->
 * diagonal (if M == s + H(i-1,j-1)); else H == Ix -> up; else H == Iy ->
 * left.  Outputs the aligned strings in forward order, the final cursor as
 * the 0-based start and end-1 as the 0-based end.
 */
static int tb_class(int c) {   /* sw.py:254-258: ord < 128 map, else -1 */
    if (c < 0 || c >= 128) return -1;
    return aa_class((uint8_t)c);
}

static int tb_sub(int a, int b) {
    int ia = tb_class(a), ib = tb_class(b);
    if (ia < 0 || ib < 0) return -5;
    return B62[ia][ib];
}

/* Returns best score; writes alignment into q_out/t_out (capacity
 * Lq+Lt+1 each), *alen, starts/ends (-1 when no alignment). */
int oracle_backtrack_affine(const uint8_t* q, int Lq, const uint8_t* t, int Lt,
                            int gap_open, int gap_extend,
                            uint8_t* q_out, uint8_t* t_out, int32_t* info) {
    /* info: [best, alen, q_start, q_end, t_start, t_end] */
    const int W = Lt + 1;
    size_t cells = (size_t)(Lq + 1) * (size_t)W;
    int16_t* M = (int16_t*)calloc(cells, sizeof(int16_t));
    int16_t* X = (int16_t*)calloc(cells, sizeof(int16_t));
    int16_t* Y = (int16_t*)calloc(cells, sizeof(int16_t));
    int16_t best = 0;
#define IDX(i, j) ((size_t)(i) * (size_t)W + (size_t)(j))
#define HV(i, j) ({ int _m = M[IDX(i, j)], _x = X[IDX(i, j)], _y = Y[IDX(i, j)]; \
                    int _h = _m; if (_x > _h) _h = _x; if (_y > _h) _h = _y;    \
                    if (_h < 0) _h = 0; _h; })
    for (int i = 1; i <= Lq; ++i) {
        for (int j = 1; j <= Lt; ++j) {
            int hd = HV(i - 1, j - 1);
            int m = tb_sub(q[i - 1], t[j - 1]) + hd;
            int hu = HV(i - 1, j);
            int xu = (i - 1 == 0) ? -16384 : X[IDX(i - 1, j)];
            int x = hu - gap_open;
            if (xu - gap_extend > x) x = xu - gap_extend;
            int hl = HV(i, j - 1);
            int yl = (j - 1 == 0) ? -16384 : Y[IDX(i, j - 1)];
            int y = hl - gap_open;
            if (yl - gap_extend > y) y = yl - gap_extend;
            M[IDX(i, j)] = (int16_t)m;
            X[IDX(i, j)] = (int16_t)x;
            Y[IDX(i, j)] = (int16_t)y;
            int h = HV(i, j);
            if (h > best) best = (int16_t)h;
        }
    }
    info[0] = best; info[1] = 0;
    info[2] = info[3] = info[4] = info[5] = -1;
    if (best > 0 && Lq > 0 && Lt > 0) {
        int ei = -1, ej = -1;
        for (int i = 1; i <= Lq && ei < 0; ++i)
            for (int j = 1; j <= Lt; ++j)
                if (HV(i, j) == best) { ei = i; ej = j; break; }
        if (ei > 0) {
            int cap = Lq + Lt + 1;
            uint8_t* qa = (uint8_t*)malloc((size_t)cap);
            uint8_t* ta = (uint8_t*)malloc((size_t)cap);
            int n = 0, ci = ei, cj = ej;
            for (int it = 0; it < Lq + Lt + 2; ++it) {
                if (ci <= 0 || cj <= 0) break;
                int h = HV(ci, cj);
                if (h == 0) break;
                int m = M[IDX(ci, cj)], x = X[IDX(ci, cj)], y = Y[IDX(ci, cj)];
                int moved = 0;
                if (h == m) {
                    int s = tb_sub(q[ci - 1], t[cj - 1]);
                    int hd = (ci > 1 && cj > 1) ? HV(ci - 1, cj - 1) : 0;
                    if (m == s + hd) {
                        qa[n] = q[ci - 1]; ta[n] = t[cj - 1];
                        ci--; cj--; moved = 1;
                    }
                } else if (h == x) {
                    int hu = (ci > 1) ? HV(ci - 1, cj) : 0;
                    int xu = (ci > 1) ? X[IDX(ci - 1, cj)] : -16384;
                    if (x == hu - gap_open || x == xu - gap_extend) {
                        qa[n] = q[ci - 1]; ta[n] = '-';
                        ci--; moved = 1;
                    }
                } else if (h == y) {
                    int hl = (cj > 1) ? HV(ci, cj - 1) : 0;
                    int yl = (cj > 1) ? Y[IDX(ci, cj - 1)] : -16384;
                    if (y == hl - gap_open || y == yl - gap_extend) {
                        qa[n] = '-'; ta[n] = t[cj - 1];
                        cj--; moved = 1;
                    }
                }
                if (!moved) break;
                n++;
            }
            for (int k = 0; k < n; ++k) {   /* forward order */
                q_out[k] = qa[n - 1 - k];
                t_out[k] = ta[n - 1 - k];
            }
            if (n > 0) {
                info[1] = n; info[2] = ci; info[3] = ei - 1;
                info[4] = cj; info[5] = ej - 1;
            }
            free(qa); free(ta);
        }
    }
#undef HV
#undef IDX
    free(M); free(X); free(Y);
    return best;
}
