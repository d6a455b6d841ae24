"""TEST INFRASTRUCTURE ONLY -- the CPU oracle for the database-search path.

This module restates the reference (AlexanderMath/sseqs 0.0.8) algorithms on
the CPU so that the CUDA product in ``sseqs_b200`` can be checked against
them.  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg import it; the product never does.

* integer work (xbit codec, Smith-Waterman, traceback) is in plain C
  (``sseqs_oracle.c``, loaded through ctypes);
* segmentation, the prefilter look-up tables, the prefilter correlation (in
  float64), selection and the a3m writer are restated here with numpy.

Each function names the reference file:line it follows.  Parity of the C
restatement is pinned against golden vectors in ``tests/golden`` (outputs of
the reference's own Triton traceback and to_a3m, and of its CUDA kernels
compiled from source by ``oracle/Makefile``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

AA = "ARNDCQEGHILKMFPSTWYV"
AA_MAP = {a: i for i, a in enumerate(AA)}

# BLOSUM62, order ARNDCQEGHILKMFPSTWYV (msa.py:110, sw.cu:7-29).
BLOSUM62 = np.array([
    [4, -1, -2, -2, 0, -1, -1, 0, -2, -1, -1, -1, -1, -2, -1, 1, 0, -3, -2, 0],
    [-1, 5, 0, -2, -3, 1, 0, -2, 0, -3, -2, 2, -1, -3, -2, -1, -1, -3, -2, -3],
    [-2, 0, 6, 1, -3, 0, 0, 0, 1, -3, -3, 0, -2, -3, -2, 1, 0, -4, -2, -3],
    [-2, -2, 1, 6, -3, 0, 2, -1, -1, -3, -4, -1, -3, -3, -1, 0, -1, -4, -3, -3],
    [0, -3, -3, -3, 9, -3, -4, -3, -3, -1, -1, -3, -1, -2, -3, -1, -1, -2, -2, -1],
    [-1, 1, 0, 0, -3, 5, 2, -2, 0, -3, -2, 1, 0, -3, -1, 0, -1, -2, -1, -2],
    [-1, 0, 0, 2, -4, 2, 5, -2, 0, -3, -3, 1, -2, -3, -1, 0, -1, -3, -2, -2],
    [0, -2, 0, -1, -3, -2, -2, 6, -2, -4, -4, -2, -3, -3, -2, 0, -2, -2, -3, -3],
    [-2, 0, 1, -1, -3, 0, 0, -2, 8, -3, -3, -1, -2, -1, -2, -1, -2, -2, 2, -3],
    [-1, -3, -3, -3, -1, -3, -3, -4, -3, 4, 2, -3, 1, 0, -3, -2, -1, -3, -1, 3],
    [-1, -2, -3, -4, -1, -2, -3, -4, -3, 2, 4, -2, 2, 0, -3, -2, -1, -2, -1, 1],
    [-1, 2, 0, -1, -3, 1, 1, -2, -1, -3, -2, 5, -1, -3, -1, 0, -1, -3, -2, -2],
    [-1, -1, -2, -3, -1, 0, -2, -3, -2, 1, 2, -1, 5, 0, -2, -1, -1, -1, -1, 1],
    [-2, -3, -3, -3, -2, -3, -3, -3, -1, 0, 0, -3, 0, 6, -4, -2, -2, 1, 3, -1],
    [-1, -2, -2, -1, -3, -1, -1, -2, -2, -3, -3, -1, -2, -4, 7, -1, -1, -4, -3, -2],
    [1, -1, 1, 0, -1, 0, 0, 0, -1, -2, -2, 0, -1, -2, -1, 4, 1, -3, -2, -2],
    [0, -1, 0, -1, -1, -1, -1, -2, -2, -1, -1, -1, -1, -2, -1, 1, 5, -2, -2, 0],
    [-3, -3, -4, -4, -2, -2, -3, -2, -2, -3, -2, -3, -1, 1, -4, -3, -2, 11, 2, -3],
    [-2, -2, -2, -3, -2, -1, -2, -3, 2, -1, -1, -2, -1, 3, -3, -2, -2, 2, 7, -1],
    [0, -3, -3, -3, -1, -2, -2, -3, -3, 3, 1, -2, 1, -1, -2, -2, 0, -3, -1, 4],
], dtype=np.int64)


def lib():
    """Load (building on first use) ``oracle/liboracle.so``."""
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "sseqs_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        i64, i32 = ctypes.c_int64, ctypes.c_int
        L.oracle_xbit_decompress.argtypes = [P, P, i64, i64]
        L.oracle_xbit_compress.argtypes = [P, P, i64]
        L.oracle_sw_linear.argtypes = [P, i32, P, i64, P, P, P, i32, i32]
        L.oracle_sw_affine.argtypes = [P, i32, P, i64, P, P, P, i32, i32, i32]
        L.oracle_backtrack_affine.argtypes = [P, i32, P, i32, i32, i32, P, P, P]
        _LIB = L
    return _LIB


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------- xbit
def xbit_compress(sym: np.ndarray) -> np.ndarray:
    """xbit.cu:36-62 / xbit_bind.cpp:11-18: u8[n] -> u8[(5n+7)//8]."""
    sym = np.ascontiguousarray(sym, dtype=np.uint8)
    out = np.zeros((sym.size * 5 + 7) // 8, dtype=np.uint8)
    lib().oracle_xbit_compress(_ptr(sym), _ptr(out), sym.size)
    return out


def xbit_decompress(packed: np.ndarray, n: int, lo: int = 0) -> np.ndarray:
    """xbit.cu:8-34 / xbit_bind.cpp:23-28: packed[lo:] -> u8[n]."""
    packed = np.ascontiguousarray(packed, dtype=np.uint8)
    need = lo + (n + 7) // 8 * 5
    if packed.size < need:   # the reference reads past the end; pad with 0
        packed = np.concatenate([packed, np.zeros(need - packed.size, np.uint8)])
    out = np.empty(n, dtype=np.uint8)
    lib().oracle_xbit_decompress(_ptr(packed), _ptr(out), n, lo)
    return out


# ------------------------------------------------------------------ SW
def encode_query(query: str) -> np.ndarray:
    """Standard residues only, as class indices (msa.py:156, sw.py:11)."""
    return np.array([AA_MAP[c] for c in query if c in AA_MAP], dtype=np.uint8)


def sw_linear(q_idx, good_idx, ascii, starts, gap=-1, nthreads=1):
    """sw_cuda_blosum62 semantics (sw.cu:55-179, sw_bind.cpp:32-73)."""
    q = np.ascontiguousarray(q_idx, dtype=np.uint8)
    g = np.ascontiguousarray(good_idx, dtype=np.int32)
    a = np.ascontiguousarray(ascii, dtype=np.uint8)
    s = np.ascontiguousarray(starts, dtype=np.int32)
    out = np.empty(g.size, dtype=np.int32)
    rc = lib().oracle_sw_linear(_ptr(q), q.size, _ptr(g), g.size, _ptr(a),
                                _ptr(s), _ptr(out), int(gap), int(nthreads))
    if rc:
        raise ValueError("query must hold class indices 0..19")
    return out


def sw_affine(q_idx, good_idx, ascii, starts, gap_open=11, gap_extend=1,
              nthreads=1):
    """sw_cuda_affine semantics (sw.cu:182-325, sw_bind.cpp:78-108)."""
    q = np.ascontiguousarray(q_idx, dtype=np.uint8)
    g = np.ascontiguousarray(good_idx, dtype=np.int32)
    a = np.ascontiguousarray(ascii, dtype=np.uint8)
    s = np.ascontiguousarray(starts, dtype=np.int32)
    out = np.empty(g.size, dtype=np.int32)
    rc = lib().oracle_sw_affine(_ptr(q), q.size, _ptr(g), g.size, _ptr(a),
                                _ptr(s), _ptr(out), int(gap_open),
                                int(gap_extend), int(nthreads))
    if rc:
        raise ValueError("query must hold class indices 0..19")
    return out


def pack_targets(targets):
    """ascii = concat(t + '@'), starts = '@' positions (sw.py:12-14)."""
    ascii = np.frombuffer("".join(t + "@" for t in targets).encode("latin-1"),
                          dtype=np.uint8).copy()
    starts = np.flatnonzero(ascii == 64).astype(np.int32)
    return ascii, starts


# ------------------------------------------------------------ traceback
def backtrack_one(query: str, target: str, gap_open=11, gap_extend=1) -> dict:
    """One target of sw_affine_backtrack (sw.py:27-219, :408-768)."""
    q = np.frombuffer(query.encode("latin-1"), dtype=np.uint8).copy()
    t = np.frombuffer(target.encode("latin-1"), dtype=np.uint8).copy()
    cap = q.size + t.size + 2
    qa = np.zeros(cap, np.uint8)
    ta = np.zeros(cap, np.uint8)
    info = np.zeros(6, np.int32)
    lib().oracle_backtrack_affine(_ptr(q) if q.size else None, q.size,
                                  _ptr(t) if t.size else None, t.size,
                                  int(gap_open), int(gap_extend),
                                  _ptr(qa), _ptr(ta), _ptr(info))
    n = int(info[1])
    return {
        "q_aligned": qa[:n].tobytes().decode("latin-1"),
        "t_aligned": ta[:n].tobytes().decode("latin-1"),
        "q_start_orig_0based": int(info[2]),
        "q_end_orig_0based": int(info[3]),
        "t_start_orig_0based": int(info[4]),
        "t_end_orig_0based": int(info[5]),
        "score": float(info[0]),
    }


def sw_affine_backtrack(query, targets, gap_open=11, gap_extend=1):
    """List form of sw.py:27-219: (best int32[B], list[dict])."""
    res = [backtrack_one(query, t, gap_open, gap_extend) for t in targets]
    return np.array([int(r["score"]) for r in res], np.int32), res


# ------------------------------------------------------------- a3m writer
def to_a3m_text(query: str, aligned: list) -> str:
    """to_a3m.py:16-72: order by score, build full-length rows, dedupe."""
    scores = [a["score"] for a in aligned]
    aligned = [aligned[i] for i in np.argsort(scores)[::-1]]

    def row(a):
        q_loc, t_loc = a["q_aligned"], a["t_aligned"]
        q_compact = q_loc.replace("-", "")
        q0 = query.find(q_compact)
        if q0 == -1:
            raise ValueError("Cannot locate aligned fragment in query.")
        mid = "".join("-" if tc == "-" else (tc.upper() if qc != "-" else tc.lower())
                      for qc, tc in zip(q_loc, t_loc))
        return "-" * q0 + mid + "-" * (len(query) - (q0 + len(q_compact)))

    out = [f">original_query\n{query}\n"]
    seen = set()
    for i, a in enumerate(aligned):
        if a["score"] == 0 or not a["q_aligned"]:
            continue
        r = row(a)
        if "@" in r or r in seen:
            continue
        seen.add(r)
        out.append(f">target_{i} score={a['score']}\n{r}\n")
    return "".join(out)


# ----------------------------------------------------------- segmentation
def segment(ascii: np.ndarray) -> dict:
    """Delimiter scan and per-segment lengths of one batch (msa.py:227-267)."""
    n = ascii.size
    delim_pos = np.flatnonzero(ascii == 64).astype(np.int64)
    starts = delim_pos + 1
    starts = starts[starts < n]
    offsets = np.concatenate([starts, [n]]).astype(np.int64)
    lengths = offsets - np.concatenate([[0], offsets[:-1]])
    lengths[:-1] -= 1
    if n and ascii[-1] == 64:
        lengths[-1] -= 1
    max_seq_length = int(lengths.max()) if lengths.size else 0
    lengths = lengths[lengths != 0]
    seg_offsets = np.zeros(lengths.size + 1, np.int64)
    seg_offsets[1:] = np.cumsum(lengths + 1)
    return {"delim_pos": delim_pos, "starts": starts, "lengths": lengths,
            "offsets": seg_offsets[:-1], "max_seq_length": max_seq_length}


# --------------------------------------------------------------- prefilter
AA_TO_POS = dict(AA_MAP)
AA_TO_POS.update({"X": 20, "-": 20, "*": 20})


def prefilter_luts(query: str, fft_rank: int = 4):
    """Query-weighted SVD of BLOSUM62 (msa.py:117-145) -> A, B f32[20, 21]."""
    b62 = BLOSUM62.copy()
    if fft_rank == 1:
        b62[b62 < 0] = 0
    w = np.sqrt(np.array([query.count(a) for a in AA]) / len(query))
    U, S, Vt = np.linalg.svd(w[:, None] * b62)
    A = np.stack([np.append(np.sqrt(s) * u, 0.0) for s, u in zip(S, U.T)])
    B = np.stack([np.append(np.sqrt(s) * v, 0.0) for s, v in zip(S, Vt)])
    return A.astype(np.float32), B.astype(np.float32)


def _db_class(ascii: np.ndarray) -> np.ndarray:
    """ASCII2POS (fft.cu:5-15): 0..19, 20 for X - *, 21 otherwise."""
    lut = np.full(256, 21, np.int64)
    for c, i in AA_TO_POS.items():
        lut[ord(c)] = i
    return lut[ascii]


def prefilter_scores(query: str, A, B, ascii, offsets, lengths, n, k=4):
    """Gapless rank-k correlation score per segment, in float64.

    fft.cu:17-415 with filter.cu:92-159 computes, in fp16, for every segment
    0.5 * max over even lags m of sum_r (a_r (*) b_r)[m], a cyclic
    convolution of length n, with a_r[i] = A_r[AA_TO_POS(query[::-1][i])]
    and b_r[i] = B_r[ASCII2POS(t[i])].  Class 21 (letters outside the 20+X
    alphabet) reads the next rank's entry 0 (fft.cu:91,124); for the last
    rank that read is past the table and is taken as 0 here.
    """
    qrev = np.array([AA_TO_POS.get(c, 20) for c in query[::-1]], np.int64)
    return prefilter_scores_codes(qrev, A, B, ascii, offsets, lengths, n, k)


def prefilter_scores_codes(qrev, A, B, ascii, offsets, lengths, n, k=4):
    """``prefilter_scores`` given the reversed query as 0..20 codes, the form
    ``warp_corr`` receives it in (sseqs/msa.py:157, filter_bind.cpp:20-64)."""
    k = max(1, min(k, A.shape[0]))
    qrev = np.asarray(qrev, np.int64)
    Lq = qrev.size
    a = np.zeros((k, n))
    a[:, :Lq] = A[:k][:, qrev]
    Bx = np.zeros((k, 22))
    Bx[:, :21] = B[:k, :21]
    for r in range(k - 1):
        Bx[r, 21] = B[r + 1, 0]
    fa = np.fft.rfft(a, n)
    out = np.zeros(len(lengths))
    cls_all = _db_class(ascii)
    for s, (off, ln) in enumerate(zip(offsets, lengths)):
        ln = min(int(ln), n)
        b = np.zeros((k, n))
        b[:, :ln] = Bx[:, cls_all[off:off + ln]]
        conv = np.fft.irfft(fa * np.fft.rfft(b, n), n).sum(0)
        out[s] = 0.5 * conv[0::2].max()
    return out


# --------------------------------------------------------------- selection
def topk_canonical(values, k):
    """Indices of the k largest values, ties broken by lower index first.

    torch.topk (msa.py:297, 324, 335) leaves the order of equal values
    unspecified; this canonical order is what parity is defined on.
    """
    values = np.asarray(values)
    order = np.lexsort((np.arange(values.size), -values.astype(np.float64)))
    return order[:k]


def search_batch(query: str, ascii: np.ndarray, *, top_fft=1, top_sw=1,
                 top_sw_affine=1000, fft_rank=4, prefilter=None):
    """One batch of msa() (msa.py:227-370) in canonical tie order.

    Returns a list of hits (segment index, affine score, linear score,
    normalised score, hit string).  ``prefilter`` supplies per-segment
    prefilter scores; None means all zero, which with top_fft=1 keeps every
    segment exactly as the reference does.
    """
    seg = segment(ascii)
    lengths = seg["lengths"]
    if lengths.size == 0:
        return []
    q_idx = encode_query(query)
    maxlen = int(lengths.max())
    scores = np.zeros(lengths.size) if prefilter is None else np.asarray(prefilter)
    k1 = lengths.size // top_fft
    cand = np.sort(topk_canonical(scores, k1))[1:-1]
    if cand.size == 0:
        return []
    delim = seg["delim_pos"].astype(np.int32)
    lin = sw_linear(q_idx, cand, ascii, delim, gap=-1, nthreads=os.cpu_count())
    k2 = lin.size // top_sw
    # msa.py:324-335 with top-k ties to the lower position: the affine
    # candidates come in the linear top-k's order (score descending), so an
    # affine tie at the cut goes to the higher linear score, then the lower
    # segment (torch.topk leaves tie order unspecified; this is the order
    # parity is defined on)
    top2 = topk_canonical(lin, k2)
    starts = seg["starts"].astype(np.int32)
    aff = sw_affine(q_idx, cand[top2], ascii, starts, 11, 1,
                    nthreads=os.cpu_count())
    if top_sw_affine > aff.size:
        raise ValueError("top_sw_affine larger than the candidate list")
    top3 = topk_canonical(aff, top_sw_affine)
    norm = (aff[top3].astype(np.float32) /
            np.sqrt(np.float32(len(query) * maxlen))).astype(np.float32)
    seg_start = np.concatenate([[0], np.cumsum(lengths[:-1] + 1)])
    hits = []
    for r, p in enumerate(top3):
        g = int(cand[top2[p]])
        st, ln = int(seg_start[g]), int(lengths[g])
        s = ascii[st:st + min(ln, 500)].tobytes().decode("latin-1")
        hits.append((g, int(aff[p]), int(lin[top2[p]]), float(norm[r]), s))
    return hits
