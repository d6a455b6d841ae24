"""a3m writer (mirrors sseqs/to_a3m.py:5-72).

Alignments come from the CUDA traceback (``sw.backtrack``) in batches of
1024 like the reference; rows are ordered with the same
``np.argsort(scores)[::-1]`` call, so for the same hit list the file is
byte-identical to the reference's.
"""
from __future__ import annotations

import numpy as np

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


def align_all(query: str, seqs: list[str], gap_open: int = 11, gap_extend: int = 1,
              batch_size: int = 1024) -> list[dict]:
    aligned: list[dict] = []
    pending = []
    for start in range(0, len(seqs), batch_size):
        pending.append(backtrack(query, list(seqs[start:start + batch_size]), gap_open, gap_extend))
    for res in pending:
        aligned.extend(res.to_dicts())
    return aligned


def to_a3m(query: str, seqs: list[str], filename: str, gap_open: int = 11, gap_extend: int = 1):
    """Write ``filename`` (sseqs/to_a3m.py:5-72)."""
    text = a3m_text(query, align_all(query, seqs, gap_open, gap_extend))
    with open(filename, "w") as f:
        f.write(text)
    return text
