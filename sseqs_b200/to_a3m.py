"""a3m writer (mirrors sseqs/to_a3m.py:5-72).

Alignments come from the CUDA traceback (``sw.backtrack``) in batches of
1024 like the reference; rows are ordered with the same
``np.argsort(scores)[::-1]`` call, so for the same hit list the file is
byte-identical to the reference's.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib, to_host
from .sw import backtrack


def a3m_text(query: str, aligned: list[dict]) -> str:
    """Build the a3m text from alignment dicts (sseqs/to_a3m.py:16-72)."""
    scores = [a["score"] for a in aligned]
    aligned = [aligned[i] for i in np.argsort(scores)[::-1]]
    parts = [f">original_query\n{query}\n"]
    seen = set()
    for i, a in enumerate(aligned):
        if a["score"] == 0 or not a["q_aligned"]:
            continue
        q_loc, t_loc = a["q_aligned"], a["t_aligned"]
        q_compact = q_loc.replace("-", "")
        q0 = query.find(q_compact)
        if q0 == -1:
            raise ValueError("Cannot locate aligned fragment in query.")
        mid = "".join("-" if tc == "-" else (tc.upper() if qc != "-" else tc.lower())
                      for qc, tc in zip(q_loc, t_loc))
        row = "-" * q0 + mid + "-" * (len(query) - (q0 + len(q_compact)))
        if "@" in row or row in seen:
            continue
        seen.add(row)
        parts.append(f">target_{i} score={a['score']}\n{row}\n")
    return "".join(parts)


def traceback_all(query: str, seqs: list[str], gap_open: int = 11, gap_extend: int = 1,
                  batch_size: int = 1024) -> list:
    """CUDA traceback of every hit, in launches of ``batch_size`` targets like
    the reference (sseqs/to_a3m.py:10-14); results stay on the device."""
    return [backtrack(query, list(seqs[start:start + batch_size]), gap_open, gap_extend)
            for start in range(0, len(seqs), batch_size)]


def align_all(query: str, seqs: list[str], gap_open: int = 11, gap_extend: int = 1,
              batch_size: int = 1024) -> list[dict]:
    return [d for res in traceback_all(query, seqs, gap_open, gap_extend, batch_size)
            for d in res.to_dicts()]


def a3m_text_raw(query: str, results: list) -> str:
    """``a3m_text`` of the traceback results ``traceback_all`` returns, with
    the row loop in the native library (``sseqs_a3m_rows``): the same rows
    in the same order (the same ``np.argsort`` of the same scores, the same
    first-occurrence placement).  Its case rule is str.upper/str.lower for
    ASCII; inputs holding other bytes take the string path of ``a3m_text``."""
    host = [(to_host(r.best), to_host(r.info), to_host(r.q_al), to_host(r.t_al), r.cap)
            for r in results]
    if not query.isascii() or any((q >= 128).any() or (t >= 128).any() for _, _, q, t, _ in host):
        return a3m_text(query, [d for r in results for d in r.to_dicts()])
    head = f">original_query\n{query}\n"
    if not host:
        return head
    scores = np.concatenate([best.astype(np.int64) for best, *_ in host])
    lens = np.ascontiguousarray(np.concatenate([info[:, 0] for _, info, *_ in host]),
                                dtype=np.int32)
    qp, tp = [], []
    for best, info, q_al, t_al, cap in host:
        start = np.arange(best.size, dtype=np.uint64) * np.uint64(cap) + \
            (np.uint64(cap) - info[:, 0].astype(np.uint64))
        qp.append(np.uint64(q_al.ctypes.data) + start)
        tp.append(np.uint64(t_al.ctypes.data) + start)
    qp, tp = np.concatenate(qp), np.concatenate(tp)
    order = np.ascontiguousarray(np.argsort(scores.astype(np.float64))[::-1], dtype=np.int64)
    qb = query.encode("ascii")
    cap_out = int(np.maximum(lens, 0).sum()) + lens.size * (len(qb) + 64) + 1
    out = np.empty(cap_out, dtype=np.uint8)
    n_out = ctypes.c_int64(0)
    st = lib().sseqs_a3m_rows(qb, len(qb), lens.size, order.ctypes.data, qp.ctypes.data,
                              tp.ctypes.data, lens.ctypes.data, scores.ctypes.data,
                              out.ctypes.data, cap_out, ctypes.byref(n_out))
    if st == 2:
        raise ValueError("Cannot locate aligned fragment in query.")
    check(st, "a3m_rows")
    return head + out[:n_out.value].tobytes().decode("ascii")


def to_a3m(query: str, seqs: list[str], filename: str, gap_open: int = 11, gap_extend: int = 1):
    """Write ``filename`` (sseqs/to_a3m.py:5-72)."""
    text = a3m_text_raw(query, traceback_all(query, seqs, gap_open, gap_extend))
    with open(filename, "w") as f:
        f.write(text)
    return text
